// Arrow C Data Interface import and export for the einfold_b200 library.
#include "arrow.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <unordered_map>

namespace ef {

Kind kind_of(const char* f) {
  if (!f) return Kind::Other;
  if (f[0] == 't' && f[1]) {
    // Temporal types: dates (tdD, tdm), times (tts, ttm, ttu, ttn),
    // timestamps (ts?:zone), durations (tD?).
    if (f[1] == 'd' && f[2] && !f[3]) return f[2] == 'D' ? Kind::Date32 : (f[2] == 'm' ? Kind::Date64 : Kind::Other);
    if (f[1] == 't' && f[2] && !f[3])
      return (f[2] == 's' || f[2] == 'm') ? Kind::Time32 : ((f[2] == 'u' || f[2] == 'n') ? Kind::Time64 : Kind::Other);
    if (f[1] == 's' && f[2] && f[3] == ':') return Kind::Timestamp;
    if (f[1] == 'D' && f[2] && !f[3]) return Kind::Duration;
    return Kind::Other;
  }
  if (f[0] == 'd' && f[1] == ':') {
    // Decimals: d:precision,scale, or d:precision,scale,bits (128 bits when
    // the bits are left out).
    int commas = 0;
    const char* bits = nullptr;
    for (const char* p = f + 2; *p; p++)
      if (*p == ',' && ++commas == 2) bits = p + 1;
    if (!bits) return commas == 1 ? Kind::Decimal128 : Kind::Other;
    if (!std::strcmp(bits, "32")) return Kind::Decimal32;
    if (!std::strcmp(bits, "64")) return Kind::Decimal64;
    if (!std::strcmp(bits, "128")) return Kind::Decimal128;
    if (!std::strcmp(bits, "256")) return Kind::Decimal256;
    return Kind::Other;
  }
  if (f[0] == 'w' && f[1] == ':') {
    // Fixed-size binary of n bytes, n > 0.
    char* end = nullptr;
    const long n = std::strtol(f + 2, &end, 10);
    return (end != f + 2 && !*end && n > 0 && n <= (1L << 20)) ? Kind::FixedBinary : Kind::Other;
  }
  if (f[0] && f[1] == 0) {
    switch (f[0]) {
      case 'c': return Kind::Int8;
      case 'C': return Kind::UInt8;
      case 's': return Kind::Int16;
      case 'S': return Kind::UInt16;
      case 'i': return Kind::Int32;
      case 'I': return Kind::UInt32;
      case 'l': return Kind::Int64;
      case 'L': return Kind::UInt64;
      case 'e': return Kind::Float16;
      case 'f': return Kind::Float32;
      case 'g': return Kind::Float64;
      case 'b': return Kind::Bool;
      case 'u': return Kind::Utf8;
      case 'U': return Kind::LargeUtf8;
      case 'z': return Kind::Binary;
      case 'Z': return Kind::LargeBinary;
      case 'n': return Kind::Null;
    }
  }
  return Kind::Other;
}

int width_of(Kind k) {
  switch (k) {
    case Kind::Int8: case Kind::UInt8: return 1;
    case Kind::Int16: case Kind::UInt16: case Kind::Float16: return 2;
    case Kind::Int32: case Kind::UInt32: case Kind::Float32: return 4;
    case Kind::Int64: case Kind::UInt64: case Kind::Float64: return 8;
    case Kind::Date32: case Kind::Time32: return 4;
    case Kind::Date64: case Kind::Time64: case Kind::Timestamp: case Kind::Duration: return 8;
    case Kind::Decimal32: return 4;
    case Kind::Decimal64: return 8;
    case Kind::Decimal128: return 16;
    case Kind::Decimal256: return 32;
    default: return 0;
  }
}

int fixed_width(const std::string& format) {
  const Kind k = kind_of(format.c_str());
  if (k == Kind::FixedBinary) return (int)std::strtol(format.c_str() + 2, nullptr, 10);
  return width_of(k);
}

const char* format_of(Kind k) {
  switch (k) {
    case Kind::Int8: return "c";
    case Kind::UInt8: return "C";
    case Kind::Int16: return "s";
    case Kind::UInt16: return "S";
    case Kind::Int32: return "i";
    case Kind::UInt32: return "I";
    case Kind::Int64: return "l";
    case Kind::UInt64: return "L";
    case Kind::Float16: return "e";
    case Kind::Float32: return "f";
    case Kind::Float64: return "g";
    case Kind::Bool: return "b";
    case Kind::Utf8: return "u";
    case Kind::LargeUtf8: return "U";
    case Kind::Binary: return "z";
    case Kind::LargeBinary: return "Z";
    case Kind::Null: return "n";
    default: return "";
  }
}

namespace {

// The cache behind pinned_acquire: free blocks by capacity (2 MiB granules),
// the capacities of blocks in use, and at most kMaxCached bytes kept free.
struct PinnedPool {
  static constexpr size_t kGranule = 2u << 20;
  static constexpr size_t kMaxCached = 16ull << 30;
  std::mutex m;
  std::multimap<size_t, void*> free_blocks;
  std::unordered_map<void*, size_t> live;
  size_t cached = 0;
};

PinnedPool& pinned_pool() {
  static PinnedPool* pool = new PinnedPool;  // outlives every result released at exit
  return *pool;
}

}  // namespace

void* pinned_acquire(size_t bytes) {
  PinnedPool& pool = pinned_pool();
  const size_t cap = (std::max<size_t>(bytes, 1) + PinnedPool::kGranule - 1) / PinnedPool::kGranule * PinnedPool::kGranule;
  {
    std::lock_guard<std::mutex> lock(pool.m);
    auto it = pool.free_blocks.lower_bound(cap);
    if (it != pool.free_blocks.end() && it->first <= 2 * cap) {
      void* p = it->second;
      pool.live[p] = it->first;
      pool.cached -= it->first;
      pool.free_blocks.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  if (cudaHostAlloc(&p, cap, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(pool.m);
  pool.live[p] = cap;
  return p;
}

void pinned_release(void* p) {
  if (!p) return;
  PinnedPool& pool = pinned_pool();
  std::lock_guard<std::mutex> lock(pool.m);
  auto it = pool.live.find(p);
  if (it == pool.live.end()) return;
  const size_t cap = it->second;
  pool.live.erase(it);
  if (pool.cached + cap > PinnedPool::kMaxCached) {
    cudaFreeHost(p);
    return;
  }
  pool.free_blocks.emplace(cap, p);
  pool.cached += cap;
}

void Buffer::reset() {
  if (ptr) {
    if (device == -2) {
      pinned_release(ptr);
    } else if (device < 0) {
      std::free(ptr);
    } else {
      int old = -1;
      cudaGetDevice(&old);
      cudaSetDevice(device);
      if (capacity) {
        // As cudaFree would: the block is free once every stream is done.
        cudaDeviceSynchronize();
        device_free_synchronized(ptr, capacity, device);
      } else {
        cudaFree(ptr);
      }
      if (old >= 0) cudaSetDevice(old);
    }
  }
  ptr = nullptr;
  bytes = 0;
  capacity = 0;
}

int64_t Column::nulls() const {
  if (!validity) return 0;
  if (null_count >= 0) return null_count;
  if (device) fail(EINFOLD_INVALID, "a device column must state its null count");
  int64_t n = 0;
  for (int64_t i = 0; i < length; i++) n += !valid(i);
  return n;
}

const uint8_t* Column::bytes(int64_t i, int64_t* len) const {
  int64_t r = offset + i;
  if (kind == Kind::LargeUtf8 || kind == Kind::LargeBinary) {
    const int64_t* o = (const int64_t*)values;
    *len = o[r + 1] - o[r];
    return data + o[r];
  }
  const int32_t* o = (const int32_t*)values;
  *len = o[r + 1] - o[r];
  return data + o[r];
}

static Field field_of(const ArrowSchema* s) {
  Field f;
  f.format = s->format ? s->format : "";
  f.name = s->name ? s->name : "";
  f.nullable = (s->flags & ARROW_FLAG_NULLABLE) != 0;
  if (s->dictionary) {
    f.dictionary = std::make_shared<Field>(field_of(s->dictionary));
    f.kind = f.dictionary->kind;  // logically the values' type
  } else {
    f.kind = kind_of(s->format);
  }
  return f;
}

std::vector<Field> import_schema(const ArrowSchema* s) {
  if (!s || !s->format || std::strcmp(s->format, "+s") != 0)
    fail(EINFOLD_INVALID, "a relation's schema must be a struct schema");
  std::vector<Field> out;
  for (int64_t i = 0; i < s->n_children; i++) out.push_back(field_of(s->children[i]));
  return out;
}

static Column column_of(const ArrowArray* a, const ArrowSchema* s, int64_t parent_offset) {
  Column c;
  c.length = a->length;
  c.offset = a->offset + parent_offset;
  c.null_count = a->null_count;
  if (s->dictionary) {
    c.index_kind = kind_of(s->format);
    c.kind = kind_of(s->dictionary->format);
    c.validity = a->n_buffers > 0 ? (const uint8_t*)a->buffers[0] : nullptr;
    c.values = a->n_buffers > 1 ? (const uint8_t*)a->buffers[1] : nullptr;
    if (!a->dictionary) fail(EINFOLD_INVALID, "a dictionary column without its dictionary");
    c.dictionary = std::make_shared<Column>(column_of(a->dictionary, s->dictionary, 0));
    return c;
  }
  c.kind = kind_of(s->format);
  if (c.kind == Kind::Null) {
    c.null_count = c.length;
    return c;
  }
  c.validity = a->n_buffers > 0 ? (const uint8_t*)a->buffers[0] : nullptr;
  c.values = a->n_buffers > 1 ? (const uint8_t*)a->buffers[1] : nullptr;
  if (is_var(c.kind)) c.data = a->n_buffers > 2 ? (const uint8_t*)a->buffers[2] : nullptr;
  if (!c.validity) c.null_count = 0;
  return c;
}

Relation import_relation(const einfold_relation* r) {
  Relation rel;
  if (!r) return rel;
  rel.fields = import_schema(r->schema);
  rel.device = r->device;
  for (int64_t i = 0; i < r->n_batches; i++) {
    const ArrowArray* b = r->batches[i];
    if (!b || b->n_children != (int64_t)rel.fields.size())
      fail(EINFOLD_INVALID, "batch %lld doesn't have the schema's %zu columns", (long long)i, rel.fields.size());
    Batch batch;
    batch.rows = b->length;
    for (int64_t c = 0; c < b->n_children; c++) {
      Column col = column_of(b->children[c], r->schema->children[c], b->offset);
      if (b->children[c]->length < b->offset + b->length)
        fail(EINFOLD_INVALID, "a column shorter than its batch");
      col.length = b->length;
      col.device = r->device >= 0;
      batch.columns.push_back(col);
    }
    rel.batches.push_back(std::move(batch));
  }
  return rel;
}

// ---- Export ----

struct ArrayPrivate {
  std::vector<OutColumn> columns;
  std::vector<ArrowArray> children;
  std::vector<ArrowArray*> child_ptrs;
  std::vector<std::vector<const void*>> child_buffers;
  std::vector<const void*> buffers;
  std::vector<ArrowArray> dicts;  // dictionary columns' values
  std::vector<std::vector<const void*>> dict_buffers;
};

static void release_child(ArrowArray* a) { a->release = nullptr; }

static void release_array(ArrowArray* a) {
  if (!a || !a->release) return;
  delete (ArrayPrivate*)a->private_data;
  a->release = nullptr;
}

static void fill_array(OutBatch&& batch, ArrowArray* out) {
  auto* p = new ArrayPrivate();
  p->columns = std::move(batch.columns);
  size_t n = p->columns.size();
  p->children.resize(n);
  p->child_ptrs.resize(n);
  p->child_buffers.resize(n);
  p->dicts.resize(n);
  p->dict_buffers.resize(n);
  auto fill = [](OutColumn& c, std::vector<const void*>& bufs, ArrowArray& a) {
    bufs.push_back(c.null_count ? c.validity.ptr : nullptr);
    bufs.push_back(c.values.ptr);
    if (is_var(c.kind)) bufs.push_back(c.data.ptr);
    std::memset(&a, 0, sizeof a);
    a.length = c.length;
    a.null_count = c.null_count;
    a.n_buffers = (int64_t)bufs.size();
    a.buffers = bufs.data();
    a.release = release_child;
  };
  for (size_t i = 0; i < n; i++) {
    OutColumn& c = p->columns[i];
    ArrowArray& a = p->children[i];
    fill(c, p->child_buffers[i], a);
    if (c.dictionary) {
      fill(*c.dictionary, p->dict_buffers[i], p->dicts[i]);
      a.dictionary = &p->dicts[i];
    }
    p->child_ptrs[i] = &a;
  }
  p->buffers.push_back(nullptr);
  std::memset(out, 0, sizeof *out);
  out->length = batch.rows;
  out->null_count = 0;
  out->n_buffers = 1;
  out->buffers = p->buffers.data();
  out->n_children = (int64_t)n;
  out->children = p->child_ptrs.data();
  out->release = release_array;
  out->private_data = p;
}

struct SchemaPrivate {
  std::vector<std::string> formats, names;
  std::vector<ArrowSchema> children;
  std::vector<ArrowSchema*> child_ptrs;
  std::vector<std::string> dict_formats;  // dictionary fields' value types
  std::vector<ArrowSchema> dicts;
};

static void release_child_schema(ArrowSchema* s) { s->release = nullptr; }

static void release_schema(ArrowSchema* s) {
  if (!s || !s->release) return;
  delete (SchemaPrivate*)s->private_data;
  s->release = nullptr;
}

void export_schema(const std::vector<Field>& fields, ArrowSchema* out) {
  auto* p = new SchemaPrivate();
  size_t n = fields.size();
  p->formats.resize(n);
  p->names.resize(n);
  p->children.resize(n);
  p->child_ptrs.resize(n);
  p->dict_formats.resize(n);
  p->dicts.resize(n);
  for (size_t i = 0; i < n; i++) {
    p->formats[i] = fields[i].format;
    p->names[i] = fields[i].name;
    ArrowSchema& s = p->children[i];
    std::memset(&s, 0, sizeof s);
    s.format = p->formats[i].c_str();
    s.name = p->names[i].c_str();
    s.flags = fields[i].nullable ? ARROW_FLAG_NULLABLE : 0;
    s.release = release_child_schema;
    if (fields[i].dictionary) {
      p->dict_formats[i] = fields[i].dictionary->format;
      ArrowSchema& d = p->dicts[i];
      std::memset(&d, 0, sizeof d);
      d.format = p->dict_formats[i].c_str();
      d.name = "";
      d.flags = ARROW_FLAG_NULLABLE;
      d.release = release_child_schema;
      s.dictionary = &d;
    }
    p->child_ptrs[i] = &s;
  }
  std::memset(out, 0, sizeof *out);
  out->format = "+s";
  out->name = "";
  out->n_children = (int64_t)n;
  out->children = p->child_ptrs.data();
  out->release = release_schema;
  out->private_data = p;
}

void export_result(std::vector<OutBatch>&& batches, const std::vector<Field>& schema, einfold_result* out) {
  out->n_batches = (int64_t)batches.size();
  out->batches = (ArrowArray*)std::calloc(batches.size() ? batches.size() : 1, sizeof(ArrowArray));
  for (size_t i = 0; i < batches.size(); i++) fill_array(std::move(batches[i]), &out->batches[i]);
  out->schema = (ArrowSchema*)std::calloc(1, sizeof(ArrowSchema));
  export_schema(schema, out->schema);
}

void release_result(einfold_result* r) {
  if (!r) return;
  if (r->batches) {
    for (int64_t i = 0; i < r->n_batches; i++)
      if (r->batches[i].release) r->batches[i].release(&r->batches[i]);
    std::free(r->batches);
    r->batches = nullptr;
  }
  if (r->schema) {
    if (r->schema->release) r->schema->release(r->schema);
    std::free(r->schema);
    r->schema = nullptr;
  }
  r->n_batches = 0;
}

// Dictionary indices of any integer type.
static int64_t read_index(const uint8_t* p, Kind k, int64_t i) {
  switch (k) {
    case Kind::Int8: return ((const int8_t*)p)[i];
    case Kind::UInt8: return ((const uint8_t*)p)[i];
    case Kind::Int16: return ((const int16_t*)p)[i];
    case Kind::UInt16: return ((const uint16_t*)p)[i];
    case Kind::Int32: return ((const int32_t*)p)[i];
    case Kind::UInt32: return ((const uint32_t*)p)[i];
    case Kind::Int64: return ((const int64_t*)p)[i];
    case Kind::UInt64: {
      const uint64_t v = ((const uint64_t*)p)[i];
      return v > (uint64_t)INT64_MAX ? -1 : (int64_t)v;
    }
    default: fail(EINFOLD_INVALID, "a dictionary whose indices aren't integers");
  }
  return -1;
}

static int64_t largest_index(Kind k) {
  switch (k) {
    case Kind::Int8: return INT8_MAX;
    case Kind::UInt8: return UINT8_MAX;
    case Kind::Int16: return INT16_MAX;
    case Kind::UInt16: return UINT16_MAX;
    case Kind::Int32: return INT32_MAX;
    case Kind::UInt32: return UINT32_MAX;
    case Kind::Int64:
    case Kind::UInt64: return INT64_MAX;
    default: fail(EINFOLD_INVALID, "a dictionary whose indices aren't integers");
  }
  return 0;
}

static void write_index(uint8_t* p, Kind k, int64_t i, int64_t v) {
  switch (k) {
    case Kind::Int8: ((int8_t*)p)[i] = (int8_t)v; break;
    case Kind::UInt8: ((uint8_t*)p)[i] = (uint8_t)v; break;
    case Kind::Int16: ((int16_t*)p)[i] = (int16_t)v; break;
    case Kind::UInt16: ((uint16_t*)p)[i] = (uint16_t)v; break;
    case Kind::Int32: ((int32_t*)p)[i] = (int32_t)v; break;
    case Kind::UInt32: ((uint32_t*)p)[i] = (uint32_t)v; break;
    default: ((int64_t*)p)[i] = v; break;
  }
}

OutColumn copy_column(const Column& c, const Field& f) {
  if (c.device) fail(EINFOLD_INVALID, "carrying a device column is not supported");
  OutColumn o;
  o.format = f.format;
  o.nullable = f.nullable;
  o.length = c.length;
  if (c.dictionary) {
    // The indices as they are, and the dictionary's values.
    if (!f.dictionary) fail(EINFOLD_INVALID, "a dictionary column of a field without a dictionary");
    o.kind = c.index_kind;
    const int w = width_of(c.index_kind);
    const int64_t nulls = c.nulls();
    o.null_count = nulls;
    if (nulls) {
      o.validity = Buffer(HostBuffer((size_t)((c.length + 7) / 8)));
      std::memset(o.validity.ptr, 0, o.validity.bytes);
      uint8_t* v = o.validity.as<uint8_t>();
      for (int64_t i = 0; i < c.length; i++)
        if (c.valid(i)) v[i >> 3] |= (uint8_t)(1u << (i & 7));
    }
    o.values = Buffer(HostBuffer((size_t)(c.length * w)));
    if (c.length) std::memcpy(o.values.ptr, c.values + c.offset * w, (size_t)(c.length * w));
    o.dictionary = std::make_shared<OutColumn>(copy_column(*c.dictionary, *f.dictionary));
    return o;
  }
  if (c.kind == Kind::Other) decline("carrying a column of type '" + f.format + "' is left to the host plan");
  o.kind = c.kind;
  int64_t nulls = c.nulls();
  o.null_count = nulls;
  if (nulls) {
    o.validity = Buffer(HostBuffer((size_t)((c.length + 7) / 8)));
    std::memset(o.validity.ptr, 0, o.validity.bytes);
    uint8_t* v = o.validity.as<uint8_t>();
    for (int64_t i = 0; i < c.length; i++)
      if (c.valid(i)) v[i >> 3] |= (uint8_t)(1u << (i & 7));
  }
  if (c.kind == Kind::Bool) {
    o.values = Buffer(HostBuffer((size_t)((c.length + 7) / 8)));
    std::memset(o.values.ptr, 0, o.values.bytes);
    uint8_t* v = o.values.as<uint8_t>();
    for (int64_t i = 0; i < c.length; i++) {
      int64_t b = c.offset + i;
      if ((c.values[b >> 3] >> (b & 7)) & 1) v[i >> 3] |= (uint8_t)(1u << (i & 7));
    }
  } else if (is_var(c.kind)) {
    bool large = c.kind == Kind::LargeUtf8 || c.kind == Kind::LargeBinary;
    int64_t total = 0;
    for (int64_t i = 0; i < c.length; i++) { int64_t l; c.bytes(i, &l); total += l; }
    o.values = Buffer(HostBuffer((size_t)(c.length + 1) * (large ? 8 : 4)));
    o.data = Buffer(HostBuffer((size_t)(total ? total : 1)));
    int64_t pos = 0;
    for (int64_t i = 0; i < c.length; i++) {
      int64_t l;
      const uint8_t* src = c.bytes(i, &l);
      if (large) o.values.as<int64_t>()[i] = pos; else o.values.as<int32_t>()[i] = (int32_t)pos;
      std::memcpy(o.data.as<uint8_t>() + pos, src, (size_t)l);
      pos += l;
    }
    if (large) o.values.as<int64_t>()[c.length] = pos; else o.values.as<int32_t>()[c.length] = (int32_t)pos;
  } else if (c.kind == Kind::Null) {
    o.null_count = c.length;
  } else {
    const int w = fixed_width(f.format);
    o.values = Buffer(HostBuffer((size_t)(c.length * w)));
    if (c.length) std::memcpy(o.values.ptr, c.values + c.offset * w, (size_t)(c.length * w));
  }
  return o;
}

// A row's value as bytes, for hashing and copying (`width` bytes of a
// fixed-width kind, or the var-length bytes).
static std::string value_bytes(const OutColumn& v, int64_t i, int width) {
  if (is_var(v.kind)) {
    const bool large = v.kind == Kind::LargeUtf8 || v.kind == Kind::LargeBinary;
    const int64_t a = large ? v.values.as<int64_t>()[i] : v.values.as<int32_t>()[i];
    const int64_t b = large ? v.values.as<int64_t>()[i + 1] : v.values.as<int32_t>()[i + 1];
    return std::string((const char*)v.data.as<uint8_t>() + a, (size_t)(b - a));
  }
  if (v.kind == Kind::Bool) return std::string(1, (char)((v.values.as<uint8_t>()[i >> 3] >> (i & 7)) & 1));
  return std::string((const char*)v.values.as<uint8_t>() + i * width, (size_t)width);
}

OutColumn dictionary_encode(OutColumn&& v, const Field& f) {
  if (!f.dictionary) fail(EINFOLD_INVALID, "dictionary_encode of a field without a dictionary");
  if (v.values.device >= 0 || v.data.device >= 0 || v.validity.device >= 0)
    fail(EINFOLD_INVALID, "dictionary-encoded key columns of results left in device memory are not supported");
  const Kind ik = kind_of(f.format.c_str());
  const int64_t cap = largest_index(ik);
  const int iw = width_of(ik);
  const int w = fixed_width(v.format);  // 0 for var-length and Bool values
  const int64_t n = v.length;
  auto valid = [&](int64_t i) { return !v.null_count || ((v.validity.as<uint8_t>()[i >> 3] >> (i & 7)) & 1); };
  // Distinct values in the order of their first rows; NULL is one of them.
  std::unordered_map<std::string, int64_t> seen;
  std::vector<int64_t> rep;  // each distinct value's first row
  int64_t null_at = -1;
  OutColumn o;
  o.format = f.format;
  o.name = v.name;
  o.nullable = f.nullable;
  o.kind = ik;
  o.length = n;
  o.values = Buffer(HostBuffer((size_t)(n ? n * iw : 1)));
  for (int64_t i = 0; i < n; i++) {
    int64_t d;
    if (!valid(i)) {
      if (null_at < 0) {
        null_at = (int64_t)rep.size();
        rep.push_back(-1);
      }
      d = null_at;
    } else {
      auto it = seen.emplace(value_bytes(v, i, w), (int64_t)rep.size());
      if (it.second) rep.push_back(i);
      d = it.first->second;
    }
    if (d > cap) fail(EINFOLD_COMPUTE, "%lld distinct keys exceed the dictionary's index type", (long long)(d + 1));
    write_index(o.values.as<uint8_t>(), ik, i, d);
  }
  auto dict = std::make_shared<OutColumn>();
  dict->format = f.dictionary->format;
  dict->kind = v.kind;
  dict->length = (int64_t)rep.size();
  const int64_t m = dict->length;
  if (null_at >= 0) {
    dict->null_count = 1;
    dict->validity = Buffer(HostBuffer((size_t)((m + 7) / 8)));
    std::memset(dict->validity.ptr, 0xff, dict->validity.bytes);
    dict->validity.as<uint8_t>()[null_at >> 3] &= (uint8_t)~(1u << (null_at & 7));
  }
  if (is_var(v.kind)) {
    const bool large = v.kind == Kind::LargeUtf8 || v.kind == Kind::LargeBinary;
    int64_t total = 0;
    for (int64_t r : rep) total += r < 0 ? 0 : (int64_t)value_bytes(v, r, 0).size();
    dict->values = Buffer(HostBuffer((size_t)(m + 1) * (large ? 8 : 4)));
    dict->data = Buffer(HostBuffer((size_t)(total ? total : 1)));
    int64_t pos = 0;
    for (int64_t j = 0; j < m; j++) {
      if (large) dict->values.as<int64_t>()[j] = pos; else dict->values.as<int32_t>()[j] = (int32_t)pos;
      if (rep[(size_t)j] < 0) continue;
      const std::string b = value_bytes(v, rep[(size_t)j], 0);
      std::memcpy(dict->data.as<uint8_t>() + pos, b.data(), b.size());
      pos += (int64_t)b.size();
    }
    if (large) dict->values.as<int64_t>()[m] = pos; else dict->values.as<int32_t>()[m] = (int32_t)pos;
  } else if (v.kind == Kind::Bool) {
    dict->values = Buffer(HostBuffer((size_t)((m + 7) / 8 ? (m + 7) / 8 : 1)));
    std::memset(dict->values.ptr, 0, dict->values.bytes);
    for (int64_t j = 0; j < m; j++)
      if (rep[(size_t)j] >= 0 && value_bytes(v, rep[(size_t)j], 0)[0])
        dict->values.as<uint8_t>()[j >> 3] |= (uint8_t)(1u << (j & 7));
  } else {
    dict->values = Buffer(HostBuffer((size_t)(m ? m * w : 1)));
    std::memset(dict->values.ptr, 0, dict->values.bytes);
    for (int64_t j = 0; j < m; j++)
      if (rep[(size_t)j] >= 0)
        std::memcpy(dict->values.as<uint8_t>() + j * w, v.values.as<uint8_t>() + rep[(size_t)j] * w, (size_t)w);
  }
  o.dictionary = std::move(dict);
  return o;
}

Relation decode_dictionaries(const Relation& r, const std::vector<int>& cols, std::vector<HostBuffer>& keep) {
  Relation out = r;
  for (int c : cols) {
    if (c < 0 || c >= (int)r.fields.size() || !r.fields[c].dictionary) continue;
    if (r.device >= 0) fail(EINFOLD_INVALID, "dictionary columns in device memory are not decoded here");
    Field vf = *r.fields[c].dictionary;
    vf.name = r.fields[c].name;
    vf.nullable = true;
    out.fields[c] = vf;
    for (size_t bi = 0; bi < r.batches.size(); bi++) {
      const Column& col = r.batches[bi].columns[c];
      if (!col.dictionary) fail(EINFOLD_INVALID, "a dictionary column without its dictionary");
      const Column& d = *col.dictionary;
      const int64_t n = col.length;
      Column nc;
      nc.kind = d.kind;
      nc.length = n;
      nc.offset = 0;
      // Each row's dictionary entry, or -1 for a NULL row.
      std::vector<int64_t> at((size_t)n);
      int64_t nulls = 0;
      for (int64_t i = 0; i < n; i++) {
        int64_t j = -1;
        if (col.valid(i)) {
          j = read_index(col.values, col.index_kind, col.offset + i);
          if (j < 0 || j >= d.length) fail(EINFOLD_INVALID, "a dictionary index out of range");
          if (!d.valid(j)) j = -1;
        }
        at[(size_t)i] = j;
        nulls += j < 0;
      }
      nc.null_count = nulls;
      if (nulls) {
        HostBuffer bits((size_t)((n + 7) / 8));
        std::memset(bits.ptr, 0, bits.bytes);
        for (int64_t i = 0; i < n; i++)
          if (at[(size_t)i] >= 0) bits.as<uint8_t>()[i >> 3] |= (uint8_t)(1u << (i & 7));
        nc.validity = bits.as<uint8_t>();
        keep.push_back(std::move(bits));
      }
      if (is_var(d.kind)) {
        const bool large = d.kind == Kind::LargeUtf8 || d.kind == Kind::LargeBinary;
        int64_t total = 0;
        for (int64_t i = 0; i < n; i++)
          if (at[(size_t)i] >= 0) {
            int64_t l;
            d.bytes(at[(size_t)i], &l);
            total += l;
          }
        if (!large && total > INT32_MAX) fail(EINFOLD_COMPUTE, "decoded dictionary keys over 2 GiB in one batch");
        HostBuffer offs((size_t)(n + 1) * (large ? 8 : 4)), data((size_t)(total ? total : 1));
        int64_t pos = 0;
        for (int64_t i = 0; i < n; i++) {
          if (large) offs.as<int64_t>()[i] = pos; else offs.as<int32_t>()[i] = (int32_t)pos;
          if (at[(size_t)i] < 0) continue;
          int64_t l;
          const uint8_t* src = d.bytes(at[(size_t)i], &l);
          std::memcpy(data.as<uint8_t>() + pos, src, (size_t)l);
          pos += l;
        }
        if (large) offs.as<int64_t>()[n] = pos; else offs.as<int32_t>()[n] = (int32_t)pos;
        nc.values = offs.as<uint8_t>();
        nc.data = data.as<uint8_t>();
        keep.push_back(std::move(offs));
        keep.push_back(std::move(data));
      } else if (d.kind == Kind::Bool) {
        HostBuffer bits((size_t)((n + 7) / 8 ? (n + 7) / 8 : 1));
        std::memset(bits.ptr, 0, bits.bytes);
        for (int64_t i = 0; i < n; i++) {
          const int64_t j = at[(size_t)i];
          if (j >= 0 && ((d.values[(d.offset + j) >> 3] >> ((d.offset + j) & 7)) & 1))
            bits.as<uint8_t>()[i >> 3] |= (uint8_t)(1u << (i & 7));
        }
        nc.values = bits.as<uint8_t>();
        keep.push_back(std::move(bits));
      } else {
        const int w = fixed_width(vf.format);
        HostBuffer vals((size_t)(n ? n * w : 1));
        std::memset(vals.ptr, 0, vals.bytes);
        for (int64_t i = 0; i < n; i++)
          if (at[(size_t)i] >= 0)
            std::memcpy(vals.as<uint8_t>() + i * w, d.values + (d.offset + at[(size_t)i]) * w, (size_t)w);
        nc.values = vals.as<uint8_t>();
        keep.push_back(std::move(vals));
      }
      out.batches[bi].columns[c] = nc;
    }
  }
  return out;
}

}  // namespace ef
