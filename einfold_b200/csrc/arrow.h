// Arrow C Data Interface: reading the caller's batches, and exporting the
// library's results as struct arrays the caller releases.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "common.h"

namespace ef {

// A column's logical type, from its Arrow format string.
// Dates, times, timestamps and durations are signed integers underneath (32
// or 64 bits) but not integer types: they rank, join and group by their
// values, and the dense and fused algorithms, which take integer keys only,
// decline them as the reference's do. Decimals (32, 64, 128 and 256 bits,
// two's complement, little-endian) rank by their values within one type, and
// fixed-size binary by its bytes; they aren't integer types either. Other: a
// type the library can't read, allowed in columns no call uses.
enum class Kind : uint8_t {
  Int8, UInt8, Int16, UInt16, Int32, UInt32, Int64, UInt64,
  Float16, Float32, Float64, Bool, Utf8, LargeUtf8, Binary, LargeBinary, Null, Other,
  Date32, Date64, Time32, Time64, Timestamp, Duration,
  Decimal32, Decimal64, Decimal128, Decimal256, FixedBinary
};

Kind kind_of(const char* format);
int width_of(Kind k);  // bytes per value of a fixed-width kind (Bool and FixedBinary: 0)
// Bytes per value of a fixed-width format, fixed-size binary (w:n) included;
// 0 for Bool, var-length and unreadable formats.
int fixed_width(const std::string& format);
inline bool is_integer(Kind k) { return k <= Kind::UInt64; }
inline bool is_signed(Kind k) { return k == Kind::Int8 || k == Kind::Int16 || k == Kind::Int32 || k == Kind::Int64; }
inline bool is_float(Kind k) { return k == Kind::Float16 || k == Kind::Float32 || k == Kind::Float64; }
inline bool is_var(Kind k) { return k == Kind::Utf8 || k == Kind::LargeUtf8 || k == Kind::Binary || k == Kind::LargeBinary; }
inline bool is_temporal(Kind k) { return k >= Kind::Date32 && k <= Kind::Duration; }
// Keys wider than 8 bytes, encoded byte by byte: 128- and 256-bit decimals
// and fixed-size binary.
inline bool is_wide(Kind k) { return k == Kind::Decimal128 || k == Kind::Decimal256 || k == Kind::FixedBinary; }
const char* format_of(Kind k);

struct Field {
  std::string format;
  std::string name;
  bool nullable = true;
  Kind kind = Kind::Other;
  std::shared_ptr<Field> dictionary;  // value type of a dictionary column
};

// A view of one column of one batch; buffers stay the caller's.
struct Column {
  Kind kind = Kind::Other;
  int64_t length = 0, offset = 0, null_count = 0;
  const uint8_t* validity = nullptr;  // bitmap, or null when every value is valid
  const uint8_t* values = nullptr;    // fixed-width values, or var-length offsets
  const uint8_t* data = nullptr;      // var-length bytes
  std::shared_ptr<Column> dictionary; // a dictionary column's values; `values` holds indices
  Kind index_kind = Kind::Other;
  bool device = false;                // buffers in device memory

  bool valid(int64_t i) const {
    if (!validity) return true;
    int64_t b = offset + i;
    return (validity[b >> 3] >> (b & 7)) & 1;
  }
  // The number of NULLs, counted when the producer left it unknown.
  int64_t nulls() const;
  // Row i as bytes (var-length kinds).
  const uint8_t* bytes(int64_t i, int64_t* len) const;
};

struct Batch {
  int64_t rows = 0;
  std::vector<Column> columns;
};

struct Relation {
  std::vector<Field> fields;
  std::vector<Batch> batches;
  int device = -1;  // -1: host memory; else the CUDA device holding the buffers
  int64_t rows() const {
    int64_t n = 0;
    for (auto& b : batches) n += b.rows;
    return n;
  }
};

std::vector<Field> import_schema(const ArrowSchema* s);
Relation import_relation(const einfold_relation* r);

// malloc'd host memory handed to an exported array.
// Page-locked host blocks for results copied from the device, from a
// process-wide cache: a released result's block serves the next result of
// a similar size, so steady-state calls neither page-lock nor touch fresh
// pages, and device-to-host copies run at the link's speed. Null when
// page-locked memory can't be had.
void* pinned_acquire(size_t bytes);
void pinned_release(void* p);

struct HostBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  bool pinned = false;  // from pinned_acquire
  HostBuffer() = default;
  explicit HostBuffer(size_t n) : ptr(n ? std::malloc(n) : nullptr), bytes(n) {
    if (n && !ptr) fail(EINFOLD_BUDGET, "out of host memory for %zu bytes", n);
  }
  // A page-locked buffer where one can be had, else an ordinary one.
  static HostBuffer page_locked(size_t n) {
    HostBuffer h;
    h.ptr = pinned_acquire(n);
    if (h.ptr) {
      h.bytes = n;
      h.pinned = true;
      return h;
    }
    return HostBuffer(n);
  }
  HostBuffer(const HostBuffer&) = delete;
  HostBuffer(HostBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes), pinned(o.pinned) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  HostBuffer& operator=(HostBuffer&& o) noexcept {
    release();
    ptr = o.ptr; bytes = o.bytes; pinned = o.pinned; o.ptr = nullptr; o.bytes = 0;
    return *this;
  }
  ~HostBuffer() { release(); }
  void release() {
    if (pinned) pinned_release(ptr);
    else std::free(ptr);
    ptr = nullptr;
  }
  template <class T> T* as() const { return (T*)ptr; }
};

// A result buffer: host memory (malloc) or device memory on `device`
// (a device_alloc block of `capacity` bytes, returned to the block cache
// after a device synchronization; cudaFree when capacity is 0).
struct Buffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  int device = -1;
  size_t capacity = 0;
  Buffer() = default;
  // device -1: host memory (malloc); -2: a page-locked block (pinned_acquire).
  Buffer(HostBuffer&& h) : ptr(h.ptr), bytes(h.bytes), device(h.pinned ? -2 : -1) { h.ptr = nullptr; h.bytes = 0; }
  Buffer(const Buffer&) = delete;
  Buffer(Buffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes), device(o.device), capacity(o.capacity) {
    o.ptr = nullptr; o.bytes = 0; o.capacity = 0;
  }
  Buffer& operator=(Buffer&& o) noexcept {
    reset();
    ptr = o.ptr; bytes = o.bytes; device = o.device; capacity = o.capacity;
    o.ptr = nullptr; o.bytes = 0; o.capacity = 0;
    return *this;
  }
  void reset();
  ~Buffer() { reset(); }
  template <class T> T* as() const { return (T*)ptr; }
};

// One column of a result: values, optional validity bitmap, and var-length data.
struct OutColumn {
  std::string format;
  std::string name;
  bool nullable = true;
  int64_t length = 0;
  int64_t null_count = 0;
  Buffer validity;  // empty when there are no NULLs
  Buffer values;
  Buffer data;      // var-length kinds only
  Kind kind = Kind::Other;
  // A dictionary column: `values` holds the indices (of `kind`), and this
  // the dictionary's values.
  std::shared_ptr<OutColumn> dictionary;
};

struct OutBatch {
  int64_t rows = 0;
  std::vector<OutColumn> columns;
};

// Exports batches (moved in) and a schema into the result.
void export_result(std::vector<OutBatch>&& batches, const std::vector<Field>& schema, einfold_result* out);
void export_schema(const std::vector<Field>& fields, ArrowSchema* out);
void release_result(einfold_result* r);

// A deep copy of rows [0, length) of a column, for carried domain columns
// (a dictionary column with its dictionary).
OutColumn copy_column(const Column& c, const Field& f);

// A host column of values as a column of the dictionary field `f`: the
// distinct values (a NULL among them once, where any row is NULL) in the
// order of their first rows, and each row's index into them.
OutColumn dictionary_encode(OutColumn&& values, const Field& f);

// `r` with its dictionary-encoded columns among `cols` replaced by their
// values, row by row (a row is NULL where its index or its value is), in
// host buffers `keep` holds. Host relations only.
Relation decode_dictionaries(const Relation& r, const std::vector<int>& cols, std::vector<HostBuffer>& keep);

}  // namespace ef
