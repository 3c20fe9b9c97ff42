// Staging Arrow columns into HBM, once per call, and small device helpers
// shared by the folds.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "arrow.h"
#include "common.h"
#include "fold.h"

namespace ef {

// One column of a relation, every batch concatenated, in HBM.
struct DeviceColumn {
  Kind kind = Kind::Other;
  int width = 0;
  int64_t rows = 0;
  int64_t nulls = 0;
  DeviceBuffer<uint8_t> data;   // fixed-width values (rows * width)
  const uint8_t* alias = nullptr;  // the caller's device buffer, used in place of `data`
  const uint8_t* ptr() const { return alias ? alias : data.get(); }
  DeviceBuffer<uint8_t> valid;  // one byte per row, 1 = valid; empty when nulls == 0
  // var-length kinds
  DeviceBuffer<int64_t> offsets;  // rows + 1
  DeviceBuffer<uint8_t> bytes;
};

// Copies column `col` of every batch into HBM; validity as bytes.
DeviceColumn stage_column(Context& ctx, const Relation& r, int col, bool with_validity = true);

// Keys of an integer column as int64, with the largest value and whether any
// is negative or too large for int64 (an unsigned 2^63 or more).
struct KeyStats {
  int64_t max = -1;
  bool negative = false;
  bool too_large = false;
};
DeviceBuffer<int64_t> keys_as_i64(Context& ctx, const DeviceColumn& c, KeyStats* stats);
// The same statistics of int64 keys already in HBM, read in place.
void key_stats_i64(Context& ctx, const int64_t* keys, int64_t n, KeyStats* stats);

// Exclusive prefix sum of n flags (uint8) into int64 positions; returns the total.
int64_t exclusive_scan_flags(Context& ctx, const uint8_t* flags, int64_t n, int64_t* out);

// Packs n bytes (0/1) into an Arrow validity bitmap of (n + 7) / 8 bytes.
void pack_bits(Context& ctx, const uint8_t* bytes, int64_t n, uint8_t* bits);

// Device to host, into a fresh host buffer.
HostBuffer to_host(Context& ctx, const void* dev, size_t bytes);

// A result buffer from a device buffer: moved into the result as it is when
// the result stays in device memory, else copied to host memory.
template <class T>
Buffer result_buffer(Context& ctx, DeviceBuffer<T>& dev, size_t bytes, bool on_device) {
  if (!on_device) return Buffer(to_host(ctx, dev.get(), bytes));
  Buffer b;
  b.ptr = dev.ptr;
  b.bytes = bytes;
  b.device = ctx.device;
  b.capacity = dev.count * sizeof(T);
  dev.ptr = nullptr;
  dev.count = 0;
  return b;
}

// A row of small descriptors passed to kernels by value.
constexpr int kMaxDims = 8;
struct Role {
  int n = 0;
  const int64_t* keys[kMaxDims] = {};
  int64_t extent[kMaxDims] = {};
};

__device__ __forceinline__ int64_t role_position(const Role& r, int64_t row) {
  int64_t p = 0;
  for (int i = 0; i < r.n; i++) p = p * r.extent[i] + r.keys[i][row];
  return p;
}

// Where output keys come from: position x (in_x) or y, their stride and extent.
struct KeyAt {
  int in_x;
  int64_t stride, extent;
  __device__ __forceinline__ int64_t at(int64_t x, int64_t y) const { return ((in_x ? x : y) / stride) % extent; }
};

// The output's key columns: where each key comes from, its width in bytes
// and its device buffer.
struct OutKeys {
  int n = 0;
  KeyAt key[kMaxDims];
  int width[kMaxDims];
  void* out[kMaxDims];
};

// The keys of output dimensions along x (or y), one table per key:
// table[k][p] = (p / stride) % extent, so that emitting needs no division.
__global__ void key_tables(int64_t n, OutKeys keys, int in_x, int64_t* __restrict__ tables);

// An int64 key narrowed to an output column of `width` bytes (Arrow's cast
// of an in-range value).
__device__ __forceinline__ void store_key(void* base, int width, int64_t i, int64_t v) {
  switch (width) {
    case 1: ((uint8_t*)base)[i] = (uint8_t)v; break;
    case 2: ((uint16_t*)base)[i] = (uint16_t)v; break;
    case 4: ((uint32_t*)base)[i] = (uint32_t)v; break;
    default: ((int64_t*)base)[i] = v; break;
  }
}

// Keys of every batch of a relation for one operand, staged as int64, with
// extents.
struct StagedKeys {
  std::vector<DeviceColumn> cols;           // staged columns (int64 ones read in place)
  std::vector<DeviceBuffer<int64_t>> wide;  // other integer columns widened to int64
  std::vector<const int64_t*> keys;         // per key of the operand, in op.keys order
  std::vector<int64_t> extent;              // per key
};

// Stages an operand's key columns; declines where dense::keys
// (crates/einfold-kernels/src/dense.rs:97-111) returns None: a key column
// that isn't integers, a NULL key, a negative one.
StagedKeys stage_keys(Context& ctx, const OperandD& op, const Relation& r);

// The keys and extents of `dims`, in order, as `op` holds them.
Role role_of(const std::vector<int>& dims, const OperandD& op, const StagedKeys& s, const std::vector<int64_t>& extent);

}  // namespace ef
