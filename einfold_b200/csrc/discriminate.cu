// The discrimination fold on the device (crates/einfold-kernels/src/discriminate.rs:369-650).
//
// 1. Keys as words. Each row's key columns are encoded into fixed-width
//    bytes that compare (as unsigned words, most significant first) in
//    Arrow's default order and are equal exactly when the host calls the keys
//    equal: per column a byte for NULL (0) or valid (1), then integers
//    sign-flipped big-endian, floats by their total-order bits (-0.0 made 0.0
//    first under SignedZerosEqual, keys.rs:61-76), strings as their bytes
//    zero-padded to the longest, then their length. A single non-NULL
//    integer column is its sign-flipped value alone (discriminate.rs:244-272).
// 2. Ranks (rank.cu): the join's keys over a‖b, the outputs' over each
//    operand with the domain's. Keys longer than four words are ranked over
//    the words that vary between keys, in rounds that refine the previous
//    round's ranks (any length, as by_bytes at :165-209).
// 3. a's joining rows sorted by (x, z, NULL-first factor bits), b's by (z, y,
//    factor bits): one stable radix sort each (the reference's two counting
//    sorts and break_ties, :497-506).
// 4. Gustavson's product, one block per output key x: its rows of a in order,
//    each adding p·q into a dense accumulator over y for the rows of b with
//    its z, in order; rows of b sharing a y are one thread's run, so every
//    group's terms are added in the reference's order, bit for bit. A first
//    traversal counts each x's groups, a second fills them, in (x, y) order.
#include <cub/cub.cuh>

#include <cmath>
#include <cstdlib>
#include <cstring>

#include "fold.h"
#include "rank.cuh"
#include "stage.cuh"

namespace ef {
namespace {

constexpr int kMaxWords = 4;  // words one ranking pass orders a key by

// One key column's block of bytes in the encoded key: a byte for NULL (0) or
// valid (1), then the value. Fixed-width values up to 8 bytes take 8, as
// order-preserving 64-bit words. 128- and 256-bit decimals take their 16 or
// 32 bytes big-endian with the sign bit flipped, fixed-size binary its bytes
// as they are, so both order bytewise as Arrow's row format orders them. A string or
// binary value takes `max_len` bytes, its own bytes zero-padded, then its
// length big-endian in `len_bytes` bytes: two values that differ first at
// byte p order by that byte, a value that is a prefix of the other with only
// zeros after it orders by its length, so the blocks order as Arrow's row
// format orders the values (bytes, a prefix first), and are equal exactly
// when the values are. Every byte's position is fixed, so any word of the key
// is computed without the bytes before it.
struct KeyCol {
  int kind;            // Kind
  int width;           // bytes of a fixed-width value
  const uint8_t* data; // fixed-width values, or var-length bytes
  const int64_t* off;  // var-length offsets
  const uint8_t* valid;
  int64_t start;       // first byte of this column's block in the key
  int64_t block;       // bytes of the block
  int64_t max_len;     // var-length: bytes of the value part
  int len_bytes;       // var-length: bytes of the length part
  int canon_zero;      // SignedZerosEqual on a float column
  int wide;            // 1: a 128/256-bit decimal, 2: fixed-size binary (bytes in the block); 0 otherwise
};

// The word positions (absolute, within the key) a pass encodes, and where
// the previous pass's ranks go (word 0) when refining.
struct WordList {
  int n = 0;
  int64_t pos[kMaxWords] = {};
};

__device__ uint64_t ordered_bits(const KeyCol& c, int64_t r) {
  switch ((Kind)c.kind) {
    case Kind::Int8: return (uint64_t)(int64_t)((const int8_t*)c.data)[r] ^ (1ull << 63);
    case Kind::Int16: return (uint64_t)(int64_t)((const int16_t*)c.data)[r] ^ (1ull << 63);
    case Kind::Int32: return (uint64_t)(int64_t)((const int32_t*)c.data)[r] ^ (1ull << 63);
    case Kind::Int64: return (uint64_t)((const int64_t*)c.data)[r] ^ (1ull << 63);
    case Kind::Date32:
    case Kind::Time32:
    case Kind::Decimal32: return (uint64_t)(int64_t)((const int32_t*)c.data)[r] ^ (1ull << 63);
    case Kind::Date64:
    case Kind::Time64:
    case Kind::Timestamp:
    case Kind::Duration:
    case Kind::Decimal64: return (uint64_t)((const int64_t*)c.data)[r] ^ (1ull << 63);
    case Kind::UInt8: return ((const uint8_t*)c.data)[r];
    case Kind::UInt16: return ((const uint16_t*)c.data)[r];
    case Kind::UInt32: return ((const uint32_t*)c.data)[r];
    case Kind::UInt64: return ((const uint64_t*)c.data)[r];
    case Kind::Bool: return c.data[r];
    case Kind::Float16: {
      uint64_t u = ((const uint16_t*)c.data)[r];
      if (c.canon_zero && u == 0x8000) u = 0;
      return ((u & 0x8000) ? (~u & 0xFFFF) : (u | 0x8000)) << 48;
    }
    case Kind::Float32: {
      uint64_t u = ((const uint32_t*)c.data)[r];
      if (c.canon_zero && u == 0x80000000u) u = 0;
      return ((u & 0x80000000u) ? (~u & 0xFFFFFFFFu) : (u | 0x80000000u)) << 32;
    }
    case Kind::Float64: {
      uint64_t u = ((const uint64_t*)c.data)[r];
      if (c.canon_zero && u == 0x8000000000000000ull) u = 0;
      return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
    }
    default: return 0;
  }
}

// Word `wpos` of row r's key (bytes 8·wpos … 8·wpos + 7, most significant first).
__device__ uint64_t key_word(const KeyCol* __restrict__ cols, int n_cols, int64_t r, int64_t wpos) {
  const int64_t b0 = wpos * 8, b1 = b0 + 8;
  uint64_t w = 0;
  for (int i = 0; i < n_cols; i++) {
    const KeyCol& c = cols[i];
    const int64_t s = c.start, e = c.start + c.block;
    if (e <= b0 || s >= b1) continue;
    const bool v = !c.valid || c.valid[r];
    const int64_t lo = s > b0 ? s : b0, hi = e < b1 ? e : b1;
    if (!v) {
      // NULL: the validity byte and everything after it are zero.
      continue;
    }
    if (c.off) {
      const int64_t o0 = c.off[r], len = c.off[r + 1] - o0;
      for (int64_t p = lo; p < hi; p++) {
        const int64_t q = p - s;
        uint64_t byte;
        if (q == 0) byte = 1;
        else if (q <= c.max_len) byte = q - 1 < len ? c.data[o0 + q - 1] : 0;
        else byte = ((uint64_t)len >> (8 * (c.len_bytes - 1 - (q - 1 - c.max_len)))) & 0xff;
        w |= byte << (8 * (7 - (p - b0)));
      }
    } else if (c.wide) {
      // Decimals: little-endian two's complement, taken most significant
      // byte first with the sign bit flipped; fixed-size binary as it is.
      const uint8_t* v = c.data + r * c.width;
      for (int64_t p = lo; p < hi; p++) {
        const int64_t q = p - s;
        uint64_t byte;
        if (q == 0) byte = 1;
        else if (c.wide == 1) byte = v[c.width - q] ^ (q == 1 ? 0x80 : 0);
        else byte = v[q - 1];
        w |= byte << (8 * (7 - (p - b0)));
      }
    } else {
      const uint64_t bits = ordered_bits(c, r);
      for (int64_t p = lo; p < hi; p++) {
        const int64_t q = p - s;
        const uint64_t byte = q == 0 ? 1 : (bits >> (8 * (8 - q))) & 0xff;
        w |= byte << (8 * (7 - (p - b0)));
      }
    }
  }
  return w;
}

// The words of `list` for rows [row0, row0 + rows), after the previous
// pass's rank (word 0) when `prefix` is given; word-major, stride ld.
__global__ void encode_words(const KeyCol* __restrict__ cols, int n_cols, int fast_int, WordList list,
                             const uint32_t* __restrict__ prefix, int64_t rows, int64_t row0,
                             uint64_t* __restrict__ out, int64_t ld) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    int o = 0;
    if (prefix) out[(int64_t)(o++) * ld + row0 + r] = prefix[row0 + r];
    if (fast_int) {
      out[(int64_t)o * ld + row0 + r] = ordered_bits(cols[0], r);
      continue;
    }
    for (int i = 0; i < list.n; i++) out[(int64_t)(o + i) * ld + row0 + r] = key_word(cols, n_cols, r, list.pos[i]);
  }
}

// For words [w0, w0 + gridDim.y) of every row: the OR and the AND over rows,
// so that words no two keys differ in are known (and skipped).
__global__ void word_spread(const KeyCol* __restrict__ cols, int n_cols, int64_t rows, int64_t w0,
                            unsigned long long* __restrict__ any, unsigned long long* __restrict__ all) {
  const int64_t wpos = w0 + blockIdx.y;
  unsigned long long o = 0, a = ~0ull;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t w = key_word(cols, n_cols, r, wpos);
    o |= w;
    a &= w;
  }
  for (int s = 16; s; s >>= 1) {
    o |= __shfl_xor_sync(0xffffffffu, o, s);
    a &= __shfl_xor_sync(0xffffffffu, a, s);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicOr(&any[blockIdx.y], o);
    atomicAnd(&all[blockIdx.y], a);
  }
}

// The longest value of a var-length column.
__global__ void longest(const int64_t* __restrict__ off, const uint8_t* __restrict__ valid, int64_t rows,
                        unsigned long long* mx) {
  unsigned long long local = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    if (valid && !valid[r]) continue;
    const unsigned long long len = (unsigned long long)(off[r + 1] - off[r]);
    local = len > local ? len : local;
  }
  for (int o = 16; o; o >>= 1) {
    unsigned long long x = __shfl_xor_sync(0xffffffffu, local, o);
    local = x > local ? x : local;
  }
  if ((threadIdx.x & 31) == 0 && local) atomicMax(mx, local);
}

// Rows with no NULL in a key compared with '=' (discriminate.rs:346-356).
__global__ void joinable_rows(int n_cols, const uint8_t* const* __restrict__ valid, const int* __restrict__ strict,
                              int64_t rows, uint8_t* __restrict__ ok) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    bool j = true;
    for (int i = 0; i < n_cols; i++)
      if (strict[i] && valid[i] && !valid[i][r]) j = false;
    ok[r] = j;
  }
}

// Sort keys of an operand's joining rows: word 0 = (major rank << 32) | minor
// rank, word 1 = factor valid (NULL first), word 2 = factor bits.
__global__ void sort_words(const int64_t* __restrict__ pick, int64_t m, const uint32_t* __restrict__ major,
                           const uint32_t* __restrict__ minor, const double* __restrict__ f,
                           const uint8_t* __restrict__ fvalid, uint64_t* __restrict__ out, int64_t ld) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = pick[i];
    const bool v = !fvalid || fvalid[r];
    out[i] = ((uint64_t)major[r] << 32) | minor[r];
    out[ld + i] = v ? 1 : 0;
    out[2 * ld + i] = v ? (uint64_t)__double_as_longlong(f[r]) : 0;
  }
}

__global__ void compact_rows(const uint8_t* __restrict__ ok, const int64_t* __restrict__ pos, int64_t rows,
                             int64_t* __restrict__ pick) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    if (ok[r]) pick[pos[r]] = r;
}

// The sorted rows' arrays: rank along `key`, factor value and validity.
__global__ void lay_out(const uint32_t* __restrict__ order, const int64_t* __restrict__ pick, int64_t m,
                        const uint32_t* __restrict__ k1, const uint32_t* __restrict__ k2, const double* __restrict__ f,
                        const uint8_t* __restrict__ fvalid, uint32_t* __restrict__ o1, uint32_t* __restrict__ o2,
                        double* __restrict__ of, uint8_t* __restrict__ ov, unsigned long long* __restrict__ count1) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = pick[order[i]];
    o1[i] = k1[r];
    o2[i] = k2[r];
    const bool v = !fvalid || fvalid[r];
    of[i] = v ? f[r] : 0.0;
    ov[i] = v;
    atomicAdd(&count1[k1[r]], 1ull);
  }
}

// Gustavson's product over x, count (fill == false) or fill (fill == true).
// acc/flags: per block, a dense accumulator over y (flags: bit 0 reached, bit 1 valued).
template <bool FILL>
__global__ void __launch_bounds__(256) gustavson(int64_t nx, int64_t ny, const int64_t* __restrict__ a_start,
                                                 const uint32_t* __restrict__ a_z, const double* __restrict__ a_f,
                                                 const uint8_t* __restrict__ a_v, const int64_t* __restrict__ b_start,
                                                 const uint32_t* __restrict__ b_y, const double* __restrict__ b_f,
                                                 const uint8_t* __restrict__ b_v, double* __restrict__ acc_all,
                                                 uint32_t* __restrict__ reached_all, uint32_t* __restrict__ valued_all,
                                                 int64_t* __restrict__ group_count, const int64_t* __restrict__ group_off,
                                                 uint32_t* __restrict__ gy, double* __restrict__ gsum,
                                                 uint8_t* __restrict__ gvalued, int64_t x_begin, int64_t x_end,
                                                 int64_t group_base) {
  const int64_t words = (ny + 31) / 32;
  double* acc = acc_all + (FILL ? (int64_t)blockIdx.x * ny : 0);
  uint32_t* reached = reached_all + (int64_t)blockIdx.x * words;
  uint32_t* valued = valued_all + (int64_t)blockIdx.x * words;
  __shared__ unsigned long long s_count;
  typedef cub::BlockScan<int, 256> BlockScanInt;
  __shared__ typename BlockScanInt::TempStorage scan_tmp;
  (void)nx;
  for (int64_t x = x_begin + blockIdx.x; x < x_end; x += gridDim.x) {
    for (int64_t i = a_start[x]; i < a_start[x + 1]; i++) {
      const uint32_t z = a_z[i];
      const double p = a_f[i];
      const bool pv = a_v[i] != 0;
      const int64_t j0 = b_start[z], j1 = b_start[z + 1];
      for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const uint32_t y = b_y[j];
        if (j > j0 && b_y[j - 1] == y) continue;  // not the first of its run
        // This thread's run: every row of b with this z and y, in order.
        bool any = false;
        double s = FILL ? acc[y] : 0.0;
        for (int64_t q = j; q < j1 && b_y[q] == y; q++) {
          if (pv && b_v[q]) {
            if (FILL) s = __dadd_rn(s, __dmul_rn(p, b_f[q]));
            any = true;
          }
        }
        const uint32_t bit = 1u << (y & 31);
        if (!(reached[y >> 5] & bit)) atomicOr(&reached[y >> 5], bit);
        if (any) {
          if (FILL) acc[y] = s;
          if (!(valued[y >> 5] & bit)) atomicOr(&valued[y >> 5], bit);
        }
      }
      __syncthreads();
    }
    // The groups of x, in y order: count, or write and clear.
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    if (!FILL) {
      unsigned long long c = 0;
      for (int64_t w = threadIdx.x; w < words; w += blockDim.x) {
        c += __popc(reached[w]);
        reached[w] = 0;
        valued[w] = 0;
      }
      atomicAdd(&s_count, c);
      __syncthreads();
      if (threadIdx.x == 0) group_count[x] = (int64_t)s_count;
    } else {
      // Ordered emission by the whole block: each thread takes a run of
      // consecutive words, a block scan of their set bits gives each run its
      // first output position, so groups come out in y order as one walk
      // would write them.
      const int64_t per = (words + blockDim.x - 1) / blockDim.x;
      const int64_t w0 = (int64_t)threadIdx.x * per, w1 = min(words, w0 + per);
      int cnt = 0;
      for (int64_t w = w0; w < w1; w++) cnt += __popc(reached[w]);
      int before;
      BlockScanInt(scan_tmp).ExclusiveSum(cnt, before);
      int64_t pos = group_off[x] - group_base + before;
      for (int64_t w = w0; w < w1; w++) {
        uint32_t bits = reached[w];
        const uint32_t vb = valued[w];
        while (bits) {
          const int k = __ffs(bits) - 1;
          bits &= bits - 1;
          const uint32_t y = (uint32_t)(w * 32 + k);
          gy[pos] = y;
          const bool v = (vb >> k) & 1u;
          gsum[pos] = v ? acc[y] : 0.0;
          gvalued[pos] = v;
          acc[y] = 0.0;
          pos++;
        }
        reached[w] = 0;
        valued[w] = 0;
      }
    }
    __syncthreads();
  }
}

__global__ void fill_x(const int64_t* __restrict__ off, int64_t x_begin, int64_t x_end, uint32_t* __restrict__ gx) {
  const int64_t base = off[x_begin];
  for (int64_t x = x_begin + blockIdx.x; x < x_end; x += gridDim.x)
    for (int64_t g = off[x] + threadIdx.x; g < off[x + 1]; g += blockDim.x) gx[g - base] = (uint32_t)x;
}

// Fixed-width gather of a key column by row (take), with validity bytes.
__global__ void gather_fixed(const uint8_t* __restrict__ data, const uint8_t* __restrict__ valid, int width,
                             int canon_zero, const uint32_t* __restrict__ first, const uint32_t* __restrict__ g,
                             int64_t n, uint8_t* __restrict__ out, uint8_t* __restrict__ ovalid,
                             unsigned long long* __restrict__ nulls) {
  unsigned long long local = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = first[g[i]];
    const bool v = !valid || valid[r];
    ovalid[i] = v;
    local += !v;
    switch (width) {
      case 1: out[i] = data[r]; break;
      case 2: ((uint16_t*)out)[i] = ((const uint16_t*)data)[r]; break;
      case 4: {
        uint32_t u = ((const uint32_t*)data)[r];
        if (canon_zero && u == 0x80000000u) u = 0;
        ((uint32_t*)out)[i] = u;
        break;
      }
      case 8: {
        uint64_t u = ((const uint64_t*)data)[r];
        if (canon_zero && u == 0x8000000000000000ull) u = 0;
        ((uint64_t*)out)[i] = u;
        break;
      }
      default:  // wide decimals and fixed-size binary
        for (int b = 0; b < width; b++) out[i * width + b] = data[r * width + b];
    }
  }
  if (local) atomicAdd(nulls, local);
}

__global__ void gather_valid(const uint8_t* __restrict__ valid, const uint32_t* __restrict__ first,
                             const uint32_t* __restrict__ g, int64_t n, uint8_t* __restrict__ ovalid,
                             unsigned long long* __restrict__ nulls) {
  unsigned long long local = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool v = !valid || valid[first[g[i]]];
    ovalid[i] = v;
    local += !v;
  }
  if (local) atomicAdd(nulls, local);
}

__global__ void gather_lengths(const int64_t* __restrict__ off, const uint32_t* __restrict__ first,
                               const uint32_t* __restrict__ g, int64_t n, int64_t* __restrict__ len) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = first[g[i]];
    len[i] = off[r + 1] - off[r];
  }
}

__global__ void gather_bytes(const uint8_t* __restrict__ data, const int64_t* __restrict__ off,
                             const uint32_t* __restrict__ first, const uint32_t* __restrict__ g,
                             const int64_t* __restrict__ out_off, int64_t n, uint8_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = first[g[i]];
    const int64_t b0 = off[r], len = off[r + 1] - b0, o = out_off[i];
    if ((((uintptr_t)(data + b0) | (uintptr_t)(out + o) | (uint64_t)len) & 7) == 0) {
      // Whole 8-byte words where the source, the destination and the length allow.
      for (int64_t b = 0; b < len; b += 8) *(uint64_t*)(out + o + b) = *(const uint64_t*)(data + b0 + b);
    } else {
      for (int64_t b = 0; b < len; b++) out[o + b] = data[b0 + b];
    }
  }
}

// Arrow Utf8/Binary offsets: the int64 offsets narrowed to int32 (the
// caller checked that the total fits).
__global__ void narrow_offsets(const int64_t* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int32_t)in[i];
}

// A domain row's value: its (x, y) group's sum when the group exists with a
// value, else the default (discriminate.rs:613-649).
__global__ void domain_lookup(int64_t rows, const uint32_t* __restrict__ xr, const uint32_t* __restrict__ yr,
                              const uint8_t* __restrict__ matches, int64_t nx, const int64_t* __restrict__ goff,
                              const uint32_t* __restrict__ gy, const double* __restrict__ gsum,
                              const uint8_t* __restrict__ gval, int has_missing, double missing,
                              double* __restrict__ val, uint8_t* __restrict__ valid) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    bool found = false;
    double v = 0.0;
    const uint32_t x = xr ? xr[r] : 0u, y = yr ? yr[r] : 0u;
    if (matches[r] && (int64_t)x < nx) {
      int64_t lo = goff[x], hi = goff[x + 1];
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (gy[mid] < y) lo = mid + 1; else hi = mid;
      }
      if (lo < goff[x + 1] && gy[lo] == y && gval[lo]) {
        found = true;
        v = gsum[lo];
      }
    }
    val[r] = found ? v : (has_missing ? missing : 0.0);
    valid[r] = found || has_missing;
  }
}

// One set of key columns from a relation (rows of every batch), staged.
struct StagedKeySet {
  std::vector<DeviceColumn> cols;
  std::vector<Kind> kinds;
  // Decoded from a dictionary: compared by bits whatever the host's float
  // keys (DataFusion takes -0.0 and 0.0 as one key in float columns, not in
  // dictionary-encoded ones; options.rs:19-22).
  std::vector<bool> dictionary;
};

// Dictionary-encoded key columns are staged as their values, row by row
// (decoded on the host; a NULL index or a NULL dictionary value is a NULL
// key), so that they rank, join and group as the plain columns of their
// values do.
StagedKeySet stage_set(Context& ctx, const Relation& r, const std::vector<int>& cols) {
  StagedKeySet s;
  bool dictionary = false;
  for (int c : cols) {
    if (c < 0 || c >= (int)r.fields.size()) fail(EINFOLD_INVALID, "no column %d", c);
    dictionary = dictionary || r.fields[c].dictionary;
    if (r.fields[c].kind == Kind::Other || (r.fields[c].dictionary && r.fields[c].dictionary->kind == Kind::Other))
      decline("keys of type '" + r.fields[c].format + "' are ranked by the host plan");
  }
  if (dictionary && r.device >= 0) decline("dictionary-encoded keys in device memory are ranked by the host plan");
  std::vector<HostBuffer> keep;
  const Relation decoded = dictionary ? decode_dictionaries(r, cols, keep) : Relation();
  const Relation& src = dictionary ? decoded : r;
  for (int c : cols) {
    s.cols.push_back(stage_column(ctx, src, c, true));
    s.kinds.push_back(src.fields[c].kind);
    s.dictionary.push_back((bool)r.fields[c].dictionary);
  }
  if (dictionary) EF_CUDA(cudaStreamSynchronize(ctx.stream));  // the decoded buffers go on return
  return s;
}

// The encoded key's layout over the rows of `sets` (the same columns' types
// each, concatenated in order), and each set's columns as the kernels read
// them.
struct KeyLayout {
  int n_cols = 0;
  bool fast = false;    // one integer column, no NULLs: its sign-flipped value alone
  int64_t bytes = 0;    // of the whole key
  int64_t words = 0;
  std::vector<DeviceBuffer<KeyCol>> cols;  // per set
};

KeyLayout layout_of(Context& ctx, const std::vector<const StagedKeySet*>& sets, int float_keys) {
  cudaStream_t s = ctx.stream;
  KeyLayout L;
  L.n_cols = sets.empty() ? 0 : (int)sets[0]->cols.size();
  const int n_cols = L.n_cols;
  L.fast = n_cols == 1 && is_integer(sets[0]->kinds[0]);
  if (L.fast)
    for (auto* st : sets) L.fast = L.fast && st->cols[0].nulls == 0;
  std::vector<int64_t> start(n_cols), block(n_cols), max_len(n_cols, 0);
  std::vector<int> len_bytes(n_cols, 0);
  for (int i = 0; i < n_cols; i++) {
    start[i] = L.bytes;
    if (is_var(sets[0]->kinds[i])) {
      DeviceBuffer<unsigned long long> dmx(1, s);
      dmx.zero();
      for (auto* st : sets) {
        const DeviceColumn& c = st->cols[i];
        if (c.rows) longest<<<blocks_for(c.rows, 256), 256, 0, s>>>(c.offsets.get(), c.valid.get(), c.rows, dmx.get());
      }
      unsigned long long mx = 0;
      EF_CUDA(cudaMemcpyAsync(&mx, dmx.get(), 8, cudaMemcpyDeviceToHost, s));
      EF_CUDA(cudaStreamSynchronize(s));
      max_len[i] = (int64_t)mx;
      while (len_bytes[i] < 8 && (mx >> (8 * len_bytes[i]))) len_bytes[i]++;
      block[i] = 1 + max_len[i] + len_bytes[i];
    } else if (is_wide(sets[0]->kinds[i])) {
      block[i] = 1 + sets[0]->cols[i].width;
    } else {
      block[i] = 1 + 8;
    }
    L.bytes += block[i];
  }
  L.words = L.fast ? 1 : std::max<int64_t>(1, (L.bytes + 7) / 8);
  for (auto* st : sets) {
    std::vector<KeyCol> kc(std::max(n_cols, 1));
    for (int i = 0; i < n_cols; i++) {
      const DeviceColumn& c = st->cols[i];
      KeyCol& k = kc[i];
      k.kind = (int)c.kind;
      k.width = c.width;
      k.data = is_var(c.kind) ? c.bytes.get() : c.ptr();
      k.off = is_var(c.kind) ? c.offsets.get() : nullptr;
      k.valid = c.valid.get();
      k.start = start[i];
      k.block = block[i];
      k.max_len = max_len[i];
      k.len_bytes = len_bytes[i];
      k.canon_zero = float_keys == 1 && is_float(c.kind) && !st->dictionary[i];
      k.wide = c.kind == Kind::FixedBinary ? 2 : (is_wide(c.kind) ? 1 : 0);
    }
    DeviceBuffer<KeyCol> d(kc.size(), s);
    EF_CUDA(cudaMemcpyAsync(d.get(), kc.data(), kc.size() * sizeof(KeyCol), cudaMemcpyHostToDevice, s));
    EF_CUDA(cudaStreamSynchronize(s));  // kc leaves scope
    L.cols.push_back(std::move(d));
  }
  return L;
}

// Writes the words of `list` (after `prefix`'s ranks as word 0, if given)
// for every row of `sets`; returns the words per key.
int encode_list(Context& ctx, const std::vector<const StagedKeySet*>& sets, const KeyLayout& L, const WordList& list,
                const uint32_t* prefix, uint64_t* out, int64_t ld) {
  cudaStream_t s = ctx.stream;
  int64_t row0 = 0;
  for (size_t i = 0; i < sets.size(); i++) {
    const int64_t rows = L.n_cols ? sets[i]->cols[0].rows : 0;
    if (rows) {
      encode_words<<<blocks_for(rows, 256), 256, 0, s>>>(L.cols[i].get(), L.n_cols, L.fast, list, prefix, rows, row0,
                                                         out, ld);
      ctx.kernels++;
    }
    row0 += rows;
  }
  EF_LAUNCH_CHECK();
  return (prefix ? 1 : 0) + (L.fast ? 1 : list.n);
}

// The positions of the words that differ between two keys, in order.
std::vector<int64_t> varying_words(Context& ctx, const std::vector<const StagedKeySet*>& sets, const KeyLayout& L) {
  cudaStream_t s = ctx.stream;
  std::vector<int64_t> out;
  constexpr int64_t kSpan = 8192;  // word positions a launch covers
  for (int64_t w0 = 0; w0 < L.words; w0 += kSpan) {
    const int64_t span = std::min(kSpan, L.words - w0);
    DeviceBuffer<unsigned long long> any((size_t)span, s), all((size_t)span, s);
    any.zero();
    EF_CUDA(cudaMemsetAsync(all.get(), 0xff, (size_t)span * 8, s));
    for (size_t i = 0; i < sets.size(); i++) {
      const int64_t rows = sets[i]->cols[0].rows;
      if (!rows) continue;
      const unsigned bx = blocks_for(rows, 256, std::max<unsigned>(1u, (unsigned)(148 * 32 / span)));
      word_spread<<<dim3(bx, (unsigned)span), 256, 0, s>>>(L.cols[i].get(), L.n_cols, rows, w0, any.get(), all.get());
      ctx.kernels++;
    }
    EF_LAUNCH_CHECK();
    std::vector<unsigned long long> ha((size_t)span), hl((size_t)span);
    EF_CUDA(cudaMemcpyAsync(ha.data(), any.get(), (size_t)span * 8, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaMemcpyAsync(hl.data(), all.get(), (size_t)span * 8, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaStreamSynchronize(s));
    for (int64_t w = 0; w < span; w++)
      if (ha[(size_t)w] != hl[(size_t)w]) out.push_back(w0 + w);
  }
  return out;
}

struct RankSet {
  DeviceBuffer<uint32_t> rank;
  DeviceBuffer<uint32_t> first;
  int64_t count = 0;
};

// The ranks of the keys of `sets` (rows concatenated) in the order of their
// bytes (discriminate.rs:212-292). Keys of up to four words are ranked in one
// radix sort. Longer keys (long strings, many columns; the reference's
// by_bytes, :165-209) are ranked over the words that differ between keys
// only, four at a time: the first sort orders the first four such words, and
// each further sort orders (the previous sort's rank, the next three words),
// which refines the ranks of the keys that agreed so far. The ranks order the
// keys as their bytes do, and the sorts are stable, so first[r] is the
// smallest row of rank r. It stops once every key has its own rank.
RankSet rank_sets(Context& ctx, const std::vector<const StagedKeySet*>& sets, int64_t total, int float_keys) {
  RankSet r;
  cudaStream_t s = ctx.stream;
  r.rank.allocate((size_t)(total ? total : 1), s);
  r.first.allocate((size_t)(total ? total : 1), s);
  if (total == 0) return r;
  const int n_cols = sets.empty() ? 0 : (int)sets[0]->cols.size();
  auto all_equal = [&]() {
    // Every key is the same: one rank, first row 0.
    EF_CUDA(cudaMemsetAsync(r.rank.get(), 0, (size_t)total * 4, s));
    EF_CUDA(cudaMemsetAsync(r.first.get(), 0, 4, s));
    r.count = 1;
  };
  if (n_cols == 0) {
    all_equal();
    return r;
  }
  KeyLayout L = layout_of(ctx, sets, float_keys);
  const int64_t ld = (total + 1) & ~(int64_t)1;
  if (L.words <= kMaxWords) {
    WordList list;
    list.n = (int)L.words;
    for (int i = 0; i < list.n; i++) list.pos[i] = i;
    DeviceBuffer<uint64_t> words((size_t)(list.n * ld), s);
    const int nw = encode_list(ctx, sets, L, list, nullptr, words.get(), ld);
    r.count = rank_keys(ctx, words.get(), nw, total, ld, r.rank.get(), r.first.get(), s);
    return r;
  }
  const std::vector<int64_t> vary = varying_words(ctx, sets, L);
  if (vary.empty()) {
    all_equal();
    return r;
  }
  DeviceBuffer<uint64_t> words((size_t)(kMaxWords * ld), s);
  DeviceBuffer<uint32_t> prev((size_t)total, s);
  size_t at = 0;
  bool refining = false;
  while (at < vary.size()) {
    WordList list;
    const int room = refining ? kMaxWords - 1 : kMaxWords;
    while (list.n < room && at < vary.size()) list.pos[list.n++] = vary[at++];
    if (refining) EF_CUDA(cudaMemcpyAsync(prev.get(), r.rank.get(), (size_t)total * 4, cudaMemcpyDeviceToDevice, s));
    const int nw = encode_list(ctx, sets, L, list, refining ? prev.get() : nullptr, words.get(), ld);
    r.count = rank_keys(ctx, words.get(), nw, total, ld, r.rank.get(), r.first.get(), s);
    refining = true;
    if (r.count == total) break;  // every key has its own rank already
  }
  return r;
}

}  // namespace

int64_t rank_columns(Context& ctx, const Relation& r, const std::vector<int>& cols, int float_keys, uint32_t* rank,
                     uint32_t* first, bool device_out) {
  cudaStream_t s = ctx.stream;
  const int64_t n = r.rows();
  if (n >= (int64_t)UINT32_MAX) fail(EINFOLD_COMPUTE, "EinFold's discrimination algorithm ranks at most 2^32 - 1 rows together");
  for (int c : cols)
    if (c < 0 || c >= (int)r.fields.size()) fail(EINFOLD_INVALID, "no column %d", c);
  StagedKeySet ks = stage_set(ctx, r, cols);
  RankSet rs = rank_sets(ctx, {&ks}, n, float_keys);
  const cudaMemcpyKind kind = device_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (n) {
    EF_CUDA(cudaMemcpyAsync(rank, rs.rank.get(), (size_t)n * 4, kind, s));
    EF_CUDA(cudaMemcpyAsync(first, rs.first.get(), (size_t)rs.count * 4, kind, s));
  }
  EF_CUDA(cudaStreamSynchronize(s));
  return rs.count;
}

FoldOutput discriminate_fold(Context& ctx, const FoldD& f, const Relation& a, const Relation& b,
                             const Relation* domain, const std::vector<Field>& schema, const einfold_options& o,
                             Budget& budget) {
  cudaStream_t s = ctx.stream;
  if (f.operands.size() != 2) fail(EINFOLD_INVALID, "the discrimination algorithm folds two operands");
  if (f.row_expr) fail(EINFOLD_COMPUTE, "row expressions are folded by the fused pipeline only");
  const int64_t na = a.rows(), nb = b.rows();
  const int64_t nd = domain ? domain->rows() : 0;
  if (std::max(na + nb, std::max(na, nb) + nd) >= (int64_t)UINT32_MAX)
    fail(EINFOLD_COMPUTE, "EinFold's discrimination algorithm ranks at most 2^32 - 1 rows together");
  const OperandD& oa = f.operands[0];
  const OperandD& ob = f.operands[1];
  std::vector<int> shared;
  for (int d = 0; d < f.n_dims(); d++)
    if (oa.holds(d) && ob.holds(d)) shared.push_back(d);
  std::vector<int> a_out, b_out;
  for (size_t i = 0; i < f.outputs.size(); i++) (oa.holds(f.outputs[i].dim) ? a_out : b_out).push_back((int)i);
  auto factor_ok = [&](const OperandD& op, const Relation& r) {
    return op.factor >= 0 && r.fields[op.factor].kind == Kind::Float64 && !r.fields[op.factor].dictionary;
  };
  if (!factor_ok(oa, a) || !factor_ok(ob, b)) fail(EINFOLD_INVALID, "factors must be Float64");
  // The reference's estimate of what ranking and ordering allocate (:414-437).
  const uint64_t ranked = sat_add(sat_mul((uint64_t)(na + nb), 2), sat_mul((uint64_t)nd, 2));
  budget.reserve(sat_add(sat_mul(ranked, 28), sat_mul((uint64_t)(na + nb), 40)), "the discrimination algorithm's ranks");

  auto cols_of = [&](const OperandD& op, const std::vector<int>& dims) {
    std::vector<int> c;
    for (int d : dims) c.push_back(op.column_of(d));
    return c;
  };
  std::vector<int> a_out_dims, b_out_dims;
  for (int i : a_out) a_out_dims.push_back(f.outputs[i].dim);
  for (int i : b_out) b_out_dims.push_back(f.outputs[i].dim);
  StagedKeySet a_sh = stage_set(ctx, a, cols_of(oa, shared)), b_sh = stage_set(ctx, b, cols_of(ob, shared));
  StagedKeySet a_o = stage_set(ctx, a, cols_of(oa, a_out_dims)), b_o = stage_set(ctx, b, cols_of(ob, b_out_dims));
  StagedKeySet d_a, d_b;
  if (domain) {
    std::vector<int> da, db;
    for (int i : a_out) da.push_back(f.outputs[i].domain_col);
    for (int i : b_out) db.push_back(f.outputs[i].domain_col);
    d_a = stage_set(ctx, *domain, da);
    d_b = stage_set(ctx, *domain, db);
  }
  ctx.phase("discriminate: staged");
  // Joinable rows: no NULL in a key compared with '='.
  auto joinable = [&](const StagedKeySet& ks, int64_t rows, DeviceBuffer<uint8_t>& ok) {
    ok.allocate((size_t)(rows ? rows : 1), s);
    std::vector<const uint8_t*> valid;
    std::vector<int> strict;
    for (size_t i = 0; i < ks.cols.size(); i++) {
      valid.push_back(ks.cols[i].valid.get());
      strict.push_back(f.equality[shared[i]] == 0);
    }
    DeviceBuffer<const uint8_t*> dv(std::max<size_t>(1, valid.size()), s);
    DeviceBuffer<int> ds(std::max<size_t>(1, strict.size()), s);
    if (!valid.empty()) {
      EF_CUDA(cudaMemcpyAsync(dv.get(), valid.data(), valid.size() * sizeof(void*), cudaMemcpyHostToDevice, s));
      EF_CUDA(cudaMemcpyAsync(ds.get(), strict.data(), strict.size() * 4, cudaMemcpyHostToDevice, s));
    }
    if (rows) joinable_rows<<<blocks_for(rows, 256), 256, 0, s>>>((int)valid.size(), dv.get(), ds.get(), rows, ok.get());
    EF_CUDA(cudaStreamSynchronize(s));
  };
  DeviceBuffer<uint8_t> a_ok, b_ok;
  joinable(a_sh, na, a_ok);
  joinable(b_sh, nb, b_ok);
  // Ranks.
  RankSet z = rank_sets(ctx, {&a_sh, &b_sh}, na + nb, o.float_keys);
  RankSet x = domain && !a_out.empty() ? rank_sets(ctx, {&a_o, &d_a}, na + nd, o.float_keys)
                                       : rank_sets(ctx, {&a_o}, na, o.float_keys);
  RankSet y = domain && !b_out.empty() ? rank_sets(ctx, {&b_o, &d_b}, nb + nd, o.float_keys)
                                       : rank_sets(ctx, {&b_o}, nb, o.float_keys);
  if (domain && a_out.empty()) {  // no a outputs: every domain row has the one rank 0
    RankSet xx;
    xx.rank.allocate((size_t)(na + nd + 1), s);
    EF_CUDA(cudaMemsetAsync(xx.rank.get(), 0, (size_t)(na + nd + 1) * 4, s));
    xx.first = std::move(x.first);
    xx.count = x.count;
    x = std::move(xx);
  }
  if (domain && b_out.empty()) {
    RankSet yy;
    yy.rank.allocate((size_t)(nb + nd + 1), s);
    EF_CUDA(cudaMemsetAsync(yy.rank.get(), 0, (size_t)(nb + nd + 1) * 4, s));
    yy.first = std::move(y.first);
    yy.count = y.count;
    y = std::move(yy);
  }
  const int64_t nx = std::max<int64_t>(x.count, 1), nz = std::max<int64_t>(z.count, 1),
                ny = std::max<int64_t>(y.count, 1);
  ctx.phase("discriminate: ranked");

  // a's joining rows by (x, z, factor bits), b's by (z, y, factor bits).
  DeviceColumn af = stage_column(ctx, a, oa.factor), bf = stage_column(ctx, b, ob.factor);
  auto order_rows = [&](int64_t rows, const DeviceBuffer<uint8_t>& ok, const uint32_t* major, const uint32_t* minor,
                        const DeviceColumn& fc, int64_t n_major, DeviceBuffer<uint32_t>& o_major,
                        DeviceBuffer<uint32_t>& o_minor, DeviceBuffer<double>& o_f, DeviceBuffer<uint8_t>& o_v,
                        DeviceBuffer<int64_t>& start) -> int64_t {
    DeviceBuffer<int64_t> pos((size_t)(rows ? rows : 1), s);
    const int64_t m = exclusive_scan_flags(ctx, ok.get(), rows, pos.get());
    DeviceBuffer<int64_t> pick((size_t)(m ? m : 1), s);
    if (rows) compact_rows<<<blocks_for(rows, 256), 256, 0, s>>>(ok.get(), pos.get(), rows, pick.get());
    const int64_t ld = (m + 1) & ~(int64_t)1;
    DeviceBuffer<uint64_t> w((size_t)(3 * ld ? 3 * ld : 1), s);
    DeviceBuffer<uint32_t> order((size_t)(m ? m : 1), s), rk((size_t)(m ? m : 1), s), fi((size_t)(m ? m : 1), s);
    o_major.allocate((size_t)(m ? m : 1), s);
    o_minor.allocate((size_t)(m ? m : 1), s);
    o_f.allocate((size_t)(m ? m : 1), s);
    o_v.allocate((size_t)(m ? m : 1), s);
    DeviceBuffer<unsigned long long> counts((size_t)n_major + 1, s);
    counts.zero();
    if (m) {
      sort_words<<<blocks_for(m, 256), 256, 0, s>>>(pick.get(), m, major, minor, (const double*)fc.ptr(),
                                                    fc.valid.get(), w.get(), ld);
      rank_keys(ctx, w.get(), 3, m, ld, rk.get(), fi.get(), s, order.get());
      lay_out<<<blocks_for(m, 256), 256, 0, s>>>(order.get(), pick.get(), m, major, minor, (const double*)fc.ptr(),
                                                 fc.valid.get(), o_major.get(), o_minor.get(), o_f.get(), o_v.get(),
                                                 counts.get());
      ctx.kernels += 3;
    }
    start.allocate((size_t)n_major + 1, s);
    EF_CUDA(cudaMemsetAsync(start.get(), 0, 8, s));
    size_t temp = 0;
    EF_CUDA(cub::DeviceScan::InclusiveSum(nullptr, temp, counts.get(), (unsigned long long*)start.get() + 1, (int)n_major, s));
    DeviceBuffer<uint8_t> t(temp ? temp : 1, s);
    EF_CUDA(cub::DeviceScan::InclusiveSum(t.get(), temp, counts.get(), (unsigned long long*)start.get() + 1, (int)n_major, s));
    EF_LAUNCH_CHECK();
    return m;
  };
  DeviceBuffer<uint32_t> a_x, a_z, b_z, b_y;
  DeviceBuffer<double> a_f, b_f;
  DeviceBuffer<uint8_t> a_v, b_v;
  DeviceBuffer<int64_t> a_start, b_start;
  const int64_t ma = order_rows(na, a_ok, x.rank.get(), z.rank.get(), af, nx, a_x, a_z, a_f, a_v, a_start);
  const int64_t mb = order_rows(nb, b_ok, z.rank.get() + na, y.rank.get(), bf, nz, b_z, b_y, b_f, b_v, b_start);
  (void)ma;
  (void)mb;
  ctx.phase("discriminate: ordered");

  // Gustavson's product: count, offsets, fill.
  const int64_t words = (ny + 31) / 32;
  // The counting pass: up to four blocks an SM, each with two bitmaps of y.
  // The filling pass: as many, but their dense accumulators and bitmaps
  // within 64 MB (at least a block an SM), so the scattered updates stay in L2.
  const uint64_t per_block = (uint64_t)(ny * 8 + words * 8);
  int count_blocks = (int)std::max<int64_t>(1, std::min<int64_t>(nx, (int64_t)ctx.sm_count * 4));
  while (count_blocks > 1 && (uint64_t)count_blocks * (uint64_t)(words * 8) > (4ull << 30)) count_blocks /= 2;
  int blocks = (int)std::min<int64_t>(
      count_blocks, std::max<int64_t>(ctx.sm_count, (int64_t)((64ull << 20) / std::max<uint64_t>(per_block, 1))));
  blocks = std::max(blocks, 1);
  while (blocks > 1 && (uint64_t)blocks * per_block > (4ull << 30)) blocks /= 2;
  budget.reserve(sat_add(sat_mul((uint64_t)blocks, (uint64_t)(ny * 8)), sat_mul((uint64_t)count_blocks, (uint64_t)(words * 8))),
                 "the discrimination algorithm's accumulators");
  DeviceBuffer<uint32_t> reached((size_t)(count_blocks * words), s), valued((size_t)(count_blocks * words), s);
  reached.zero();
  valued.zero();
  DeviceBuffer<int64_t> gcount((size_t)nx, s), goff((size_t)nx + 1, s);
  gustavson<false><<<count_blocks, 256, 0, s>>>(nx, ny, a_start.get(), a_z.get(), a_f.get(), a_v.get(), b_start.get(),
                                          b_y.get(), b_f.get(), b_v.get(), nullptr, reached.get(), valued.get(),
                                          gcount.get(), nullptr, nullptr, nullptr, nullptr, 0, nx, 0);
  ctx.kernels++;
  EF_LAUNCH_CHECK();
  EF_CUDA(cudaMemsetAsync(goff.get(), 0, 8, s));
  {
    size_t temp = 0;
    EF_CUDA(cub::DeviceScan::InclusiveSum(nullptr, temp, gcount.get(), goff.get() + 1, (int)nx, s));
    DeviceBuffer<uint8_t> t(temp ? temp : 1, s);
    EF_CUDA(cub::DeviceScan::InclusiveSum(t.get(), temp, gcount.get(), goff.get() + 1, (int)nx, s));
  }
  int64_t groups = 0;
  EF_CUDA(cudaMemcpyAsync(&groups, goff.get() + nx, 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  const uint64_t out_bytes = f.domain ? (uint64_t)nd * 8 : sat_mul((uint64_t)groups, 8 * (f.outputs.size() + 1));
  budget.reserve(sat_add(sat_mul((uint64_t)groups, 24), out_bytes), "the discrimination algorithm's groups");
  DeviceBuffer<double> acc((size_t)blocks * ny, s);
  acc.zero();
  // The groups of x in [x_begin, x_end), in (x, y) order, into arrays of
  // their own (the accumulators and bitmaps are left cleared for the next).
  auto fill = [&](int64_t x_begin, int64_t x_end, uint32_t* gy, double* gsum, uint8_t* gval, int64_t base) {
    gustavson<true><<<blocks, 256, 0, s>>>(nx, ny, a_start.get(), a_z.get(), a_f.get(), a_v.get(), b_start.get(),
                                           b_y.get(), b_f.get(), b_v.get(), acc.get(), reached.get(), valued.get(),
                                           nullptr, goff.get(), gy, gsum, gval, x_begin, x_end, base);
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  };

  FoldOutput result;
  result.algorithm = EINFOLD_ALG_DISCRIMINATE;
  if (f.domain) {
    DeviceBuffer<uint32_t> gy((size_t)(groups ? groups : 1), s);
    DeviceBuffer<double> gsum((size_t)(groups ? groups : 1), s);
    DeviceBuffer<uint8_t> gval((size_t)(groups ? groups : 1), s);
    fill(0, nx, gy.get(), gsum.get(), gval.get(), 0);
    ctx.phase("discriminate: product");
    if (!domain) fail(EINFOLD_INVALID, "a fold with a domain was given no domain relation");
    if (o.result_on_device) fail(EINFOLD_INVALID, "results in device memory are not supported with a domain");
    const DomainD& spec = *f.domain;
    // Domain rows joinable under each output's domain equality.
    std::vector<int> all_cols;
    for (auto& out : f.outputs) all_cols.push_back(out.domain_col);
    StagedKeySet dk = stage_set(ctx, *domain, all_cols);
    DeviceBuffer<uint8_t> matches((size_t)(nd ? nd : 1), s);
    {
      std::vector<const uint8_t*> valid;
      std::vector<int> strict;
      for (size_t i = 0; i < f.outputs.size(); i++) {
        valid.push_back(dk.cols[i].valid.get());
        strict.push_back(f.outputs[i].domain_eq == 0);
      }
      DeviceBuffer<const uint8_t*> dv(std::max<size_t>(1, valid.size()), s);
      DeviceBuffer<int> ds(std::max<size_t>(1, strict.size()), s);
      if (!valid.empty()) {
        EF_CUDA(cudaMemcpyAsync(dv.get(), valid.data(), valid.size() * sizeof(void*), cudaMemcpyHostToDevice, s));
        EF_CUDA(cudaMemcpyAsync(ds.get(), strict.data(), strict.size() * 4, cudaMemcpyHostToDevice, s));
      }
      if (nd) joinable_rows<<<blocks_for(nd, 256), 256, 0, s>>>((int)valid.size(), dv.get(), ds.get(), nd, matches.get());
    }
    DeviceBuffer<double> val((size_t)(nd ? nd : 1), s);
    DeviceBuffer<uint8_t> valid((size_t)(nd ? nd : 1), s);
    if (nd)
      domain_lookup<<<blocks_for(nd, 256), 256, 0, s>>>(nd, x.rank.get() + na, y.rank.get() + nb, matches.get(), nx,
                                                        goff.get(), gy.get(), gsum.get(), gval.get(), spec.has_missing,
                                                        spec.missing, val.get(), valid.get());
    EF_LAUNCH_CHECK();
    HostBuffer hv = to_host(ctx, val.get(), (size_t)nd * 8);
    HostBuffer hvalid = to_host(ctx, valid.get(), (size_t)nd);
    int64_t off = 0;
    for (auto& batch : domain->batches) {
      OutBatch ob2;
      ob2.rows = batch.rows;
      for (size_t i = 0; i < spec.carry.size(); i++) {
        OutColumn c = copy_column(batch.columns[spec.carry[i]], domain->fields[spec.carry[i]]);
        c.format = schema[i].format;
        c.name = schema[i].name;
        ob2.columns.push_back(std::move(c));
      }
      OutColumn v;
      v.format = "g";
      v.kind = Kind::Float64;
      v.name = schema.back().name;
      v.length = batch.rows;
      v.values = Buffer(HostBuffer((size_t)batch.rows * 8));
      if (batch.rows) std::memcpy(v.values.ptr, hv.as<double>() + off, (size_t)batch.rows * 8);
      int64_t nulls = 0;
      for (int64_t i = 0; i < batch.rows; i++) nulls += !hvalid.as<uint8_t>()[off + i];
      v.null_count = nulls;
      if (nulls) {
        v.validity = Buffer(HostBuffer((size_t)(batch.rows + 7) / 8));
        std::memset(v.validity.ptr, 0, v.validity.bytes);
        for (int64_t i = 0; i < batch.rows; i++)
          if (hvalid.as<uint8_t>()[off + i]) v.validity.as<uint8_t>()[i >> 3] |= (uint8_t)(1u << (i & 7));
      }
      ob2.columns.push_back(std::move(v));
      result.batches.push_back(std::move(ob2));
      off += batch.rows;
    }
    return result;
  }

  // The result in batches of at most EINFOLD_GROUPS_PER_BATCH groups (2^28
  // by default): the groups of consecutive x blocks, each batch's product,
  // keys and values computed, copied out and freed before the next, so that
  // device memory holds one batch's groups at a time however many the fold
  // makes. x blocks are independent (discriminate.rs:548-584), and the
  // batches come out in (x, y) order.
  static const int64_t per_batch = [] {
    const char* e = std::getenv("EINFOLD_GROUPS_PER_BATCH");
    const long long v = e ? std::atoll(e) : (1ll << 28);
    return (int64_t)std::max(1ll, v);
  }();
  std::vector<int64_t> hoff((size_t)nx + 1);
  EF_CUDA(cudaMemcpyAsync(hoff.data(), goff.get(), (size_t)(nx + 1) * 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  int64_t x_begin = 0;
  do {
    int64_t x_end = x_begin + 1;
    while (x_end < nx && hoff[(size_t)x_end + 1] - hoff[(size_t)x_begin] <= per_batch) x_end++;
    if (nx == 0) x_end = 0;
    const int64_t base = nx ? hoff[(size_t)x_begin] : 0;
    const int64_t groups = nx ? hoff[(size_t)x_end] - base : 0;
    DeviceBuffer<uint32_t> gy((size_t)(groups ? groups : 1), s), gx((size_t)(groups ? groups : 1), s);
    DeviceBuffer<double> gsum((size_t)(groups ? groups : 1), s);
    DeviceBuffer<uint8_t> gval((size_t)(groups ? groups : 1), s);
    if (groups) fill(x_begin, x_end, gy.get(), gsum.get(), gval.get(), base);
    ctx.phase("discriminate: product");
    // Groups' keys from a row of a or b that has them (take of first rows).
    if (groups) {
      fill_x<<<std::max<int64_t>(1, std::min<int64_t>(x_end - x_begin, 65535)), 256, 0, s>>>(goff.get(), x_begin,
                                                                                            x_end, gx.get());
      ctx.kernels++;
    }
    OutBatch out_batch;
    out_batch.rows = groups;
    for (size_t i = 0; i < f.outputs.size(); i++) {
      const bool from_a = oa.holds(f.outputs[i].dim);
      const std::vector<int>& outs = from_a ? a_out : b_out;
      size_t j = 0;
      while (outs[j] != (int)i) j++;
      const DeviceColumn& src = (from_a ? a_o : b_o).cols[j];
      const bool src_dict = (from_a ? a_o : b_o).dictionary[j];
      const uint32_t* first = from_a ? x.first.get() : y.first.get();
      const uint32_t* g = from_a ? gx.get() : gy.get();
      OutColumn c;
      c.format = schema[i].format;
      c.name = schema[i].name;
      c.kind = schema[i].kind;
      c.nullable = schema[i].nullable;
      c.length = groups;
      DeviceBuffer<uint8_t> cvalid((size_t)(groups ? groups : 1), s);
      DeviceBuffer<unsigned long long> cn(1, s);
      cn.zero();
      if (is_var(src.kind)) {
        DeviceBuffer<int64_t> len((size_t)(groups ? groups : 1), s), offs((size_t)groups + 1, s);
        if (groups) {
          gather_lengths<<<blocks_for(groups, 256), 256, 0, s>>>(src.offsets.get(), first, g, groups, len.get());
          EF_CUDA(cudaMemsetAsync(offs.get(), 0, 8, s));
          size_t temp = 0;
          EF_CUDA(cub::DeviceScan::InclusiveSum(nullptr, temp, len.get(), offs.get() + 1, (int)groups, s));
          DeviceBuffer<uint8_t> t(temp ? temp : 1, s);
          EF_CUDA(cub::DeviceScan::InclusiveSum(t.get(), temp, len.get(), offs.get() + 1, (int)groups, s));
        } else {
          EF_CUDA(cudaMemsetAsync(offs.get(), 0, 8, s));
        }
        int64_t total = 0;
        EF_CUDA(cudaMemcpyAsync(&total, offs.get() + groups, 8, cudaMemcpyDeviceToHost, s));
        EF_CUDA(cudaStreamSynchronize(s));
        DeviceBuffer<uint8_t> bytes((size_t)(total ? total : 1), s);
        if (groups) {
          gather_bytes<<<blocks_for(groups, 256), 256, 0, s>>>(src.bytes.get(), src.offsets.get(), first, g, offs.get(),
                                                               groups, bytes.get());
          gather_valid<<<blocks_for(groups, 256), 256, 0, s>>>(src.valid.get(), first, g, groups, cvalid.get(), cn.get());
        }
        const bool large = src.kind == Kind::LargeUtf8 || src.kind == Kind::LargeBinary;
        if (large) {
          c.values = result_buffer(ctx, offs, (size_t)(groups + 1) * 8, o.result_on_device);
        } else {
          if (total > INT32_MAX) fail(EINFOLD_COMPUTE, "string output over 2 GiB");
          DeviceBuffer<int32_t> o32((size_t)groups + 1, s);
          narrow_offsets<<<blocks_for((uint64_t)groups + 1, 256), 256, 0, s>>>(offs.get(), groups + 1, o32.get());
          ctx.kernels++;
          c.values = result_buffer(ctx, o32, (size_t)(groups + 1) * 4, o.result_on_device);
        }
        c.data = result_buffer(ctx, bytes, (size_t)total, o.result_on_device);
      } else {
        const int width = src.width ? src.width : 1;
        DeviceBuffer<uint8_t> vals((size_t)(groups ? groups * width : 1), s);
        if (groups)
          gather_fixed<<<blocks_for(groups, 256), 256, 0, s>>>(src.ptr(), src.valid.get(), width,
                                                               o.float_keys == 1 && is_float(src.kind) && !src_dict,
                                                               first, g, groups,
                                                               vals.get(), cvalid.get(), cn.get());
        c.values = result_buffer(ctx, vals, (size_t)(groups * width), o.result_on_device);
      }
      unsigned long long cnulls = 0;
      EF_CUDA(cudaMemcpyAsync(&cnulls, cn.get(), 8, cudaMemcpyDeviceToHost, s));
      EF_CUDA(cudaStreamSynchronize(s));
      c.null_count = (int64_t)cnulls;
      if (cnulls) {
        DeviceBuffer<uint8_t> bits((size_t)((groups + 7) / 8), s);
        pack_bits(ctx, cvalid.get(), groups, bits.get());
        c.validity = result_buffer(ctx, bits, (size_t)((groups + 7) / 8), o.result_on_device);
      }
      if (schema[i].dictionary) {
        // A dictionary-encoded key: the gathered values, encoded again.
        c.format = schema[i].dictionary->format;
        c = dictionary_encode(std::move(c), schema[i]);
      }
      out_batch.columns.push_back(std::move(c));
    }
    OutColumn v;
    v.format = "g";
    v.kind = Kind::Float64;
    v.name = schema.back().name;
    v.length = groups;
    DeviceBuffer<uint8_t> vbits((size_t)((groups + 7) / 8 ? (groups + 7) / 8 : 1), s);
    unsigned long long vnulls = 0;
    {
      DeviceBuffer<unsigned long long> cnt(1, s);
      cnt.zero();
      // NULL where no product had a value.
      DeviceBuffer<uint8_t> inv((size_t)(groups ? groups : 1), s);
      if (groups) {
        pack_bits(ctx, gval.get(), groups, vbits.get());
        size_t temp = 0;
        cub::TransformInputIterator<unsigned long long, cub::CastOp<unsigned long long>, const uint8_t*> it(
            gval.get(), cub::CastOp<unsigned long long>());
        EF_CUDA(cub::DeviceReduce::Sum(nullptr, temp, it, cnt.get(), (int)groups, s));
        DeviceBuffer<uint8_t> t(temp ? temp : 1, s);
        EF_CUDA(cub::DeviceReduce::Sum(t.get(), temp, it, cnt.get(), (int)groups, s));
        unsigned long long valued_n = 0;
        EF_CUDA(cudaMemcpyAsync(&valued_n, cnt.get(), 8, cudaMemcpyDeviceToHost, s));
        EF_CUDA(cudaStreamSynchronize(s));
        vnulls = (unsigned long long)groups - valued_n;
      }
    }
    v.values = result_buffer(ctx, gsum, (size_t)groups * 8, o.result_on_device);
    v.null_count = (int64_t)vnulls;
    if (vnulls) v.validity = result_buffer(ctx, vbits, (size_t)((groups + 7) / 8), o.result_on_device);
    out_batch.columns.push_back(std::move(v));
    EF_CUDA(cudaStreamSynchronize(s));
    result.batches.push_back(std::move(out_batch));
    x_begin = x_end;
  } while (x_begin < nx);
  ctx.phase("discriminate: result");
  return result;
}

}  // namespace ef
