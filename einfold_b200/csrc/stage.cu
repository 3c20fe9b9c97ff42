// Staging Arrow columns into HBM, and the scan/pack helpers.
#include <cub/cub.cuh>

#include "stage.cuh"

namespace ef {
namespace {

struct Segment {
  int64_t row;       // first row of the batch in the concatenation
  int64_t byte;      // where its bitmap bytes start in the staged bitmap
  int32_t shift;     // bit of its first row in the first byte
  int32_t pad;
};

__global__ void expand_validity(const uint8_t* __restrict__ bits, const Segment* __restrict__ seg, int n_seg,
                                int64_t rows, uint8_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = n_seg - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (seg[mid].row <= i) lo = mid; else hi = mid - 1;
    }
    const Segment s = seg[lo];
    if (s.byte < 0) { out[i] = 1; continue; }
    const int64_t b = (int64_t)s.shift + (i - s.row);
    out[i] = (bits[s.byte + (b >> 3)] >> (b & 7)) & 1;
  }
}

template <class T>
__global__ void widen(const T* __restrict__ in, int64_t n, int64_t* __restrict__ out, unsigned long long* max,
                      int* flags) {
  int64_t local = -1;
  int f = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    T v = in[i];
    int64_t w;
    if constexpr (sizeof(T) == 8 && !std::is_signed<T>::value) {
      if ((uint64_t)v >= (1ull << 63)) { f |= 2; w = -1; } else w = (int64_t)v;
    } else {
      w = (int64_t)v;
    }
    if (w < 0) f |= 1;
    if (out) out[i] = w;
    if (w > local) local = w;
  }
  for (int o = 16; o; o >>= 1) {
    long long other = __shfl_xor_sync(0xffffffffu, (long long)local, o);
    if (other > local) local = other;
    f |= __shfl_xor_sync(0xffffffffu, f, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (local >= 0) atomicMax(max, (unsigned long long)local);
    if (f) atomicOr(flags, f);
  }
}

__global__ void pack_bits_kernel(const uint8_t* __restrict__ in, int64_t n, uint8_t* __restrict__ out) {
  const int64_t bytes = (n + 7) / 8;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < bytes; i += (int64_t)gridDim.x * blockDim.x) {
    uint8_t v = 0;
    for (int j = 0; j < 8; j++) {
      const int64_t r = i * 8 + j;
      if (r < n && in[r]) v |= (uint8_t)(1u << j);
    }
    out[i] = v;
  }
}

}  // namespace

DeviceColumn stage_column(Context& ctx, const Relation& r, int col, bool with_validity) {
  DeviceColumn d;
  cudaStream_t s = ctx.stream;
  if (col < 0 || col >= (int)r.fields.size()) fail(EINFOLD_INVALID, "column %d of a relation with %zu", col, r.fields.size());
  d.kind = r.fields[col].kind;
  d.rows = r.rows();
  const cudaMemcpyKind from = r.device >= 0 ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (r.device >= 0 && r.device != ctx.device)
    fail(EINFOLD_INVALID, "a relation on device %d given to a context on device %d", r.device, ctx.device);
  for (auto& b : r.batches) {
    const Column& c = b.columns[col];
    if (c.dictionary) fail(EINFOLD_INVALID, "dictionary columns are not staged here");
    d.nulls += c.nulls();
  }
  if (is_var(d.kind)) {
    if (r.device >= 0) fail(EINFOLD_INVALID, "variable-length columns must be in host memory");
    bool large = d.kind == Kind::LargeUtf8 || d.kind == Kind::LargeBinary;
    // Offsets rebased per batch on the host (one pass over the offsets), bytes copied as they are.
    std::vector<int64_t> off((size_t)d.rows + 1);
    int64_t total = 0, row = 0;
    std::vector<std::pair<const uint8_t*, int64_t>> spans;
    for (auto& b : r.batches) {
      const Column& c = b.columns[col];
      if (c.length == 0) continue;
      int64_t first, last;
      if (large) { first = ((const int64_t*)c.values)[c.offset]; last = ((const int64_t*)c.values)[c.offset + c.length]; }
      else { first = ((const int32_t*)c.values)[c.offset]; last = ((const int32_t*)c.values)[c.offset + c.length]; }
      for (int64_t i = 0; i < c.length; i++) {
        int64_t o = large ? ((const int64_t*)c.values)[c.offset + i] : ((const int32_t*)c.values)[c.offset + i];
        off[(size_t)(row + i)] = total + (o - first);
      }
      spans.push_back({c.data + first, last - first});
      total += last - first;
      row += c.length;
    }
    off[(size_t)d.rows] = total;
    d.offsets.allocate((size_t)d.rows + 1, s);
    EF_CUDA(cudaMemcpyAsync(d.offsets.get(), off.data(), off.size() * 8, cudaMemcpyHostToDevice, s));
    d.bytes.allocate((size_t)(total ? total : 1), s);
    int64_t pos = 0;
    for (auto& sp : spans) {
      if (sp.second) EF_CUDA(cudaMemcpyAsync(d.bytes.get() + pos, sp.first, (size_t)sp.second, cudaMemcpyHostToDevice, s));
      pos += sp.second;
    }
    EF_CUDA(cudaStreamSynchronize(s));  // `off` is a host temporary
  } else if (d.kind == Kind::Bool) {
    // Booleans are bit-packed; expanded to bytes with the validity machinery.
    d.width = 1;
    d.data.allocate((size_t)(d.rows ? d.rows : 1), s);
    std::vector<Segment> seg;
    int64_t nbytes = 0, row = 0;
    for (auto& b : r.batches) {
      const Column& c = b.columns[col];
      int64_t first = c.offset / 8, last = (c.offset + c.length + 7) / 8;
      seg.push_back({row, nbytes, (int32_t)(c.offset % 8), 0});
      nbytes += last - first;
      row += c.length;
    }
    DeviceBuffer<uint8_t> bits((size_t)(nbytes ? nbytes : 1), s);
    int64_t pos = 0;
    for (auto& b : r.batches) {
      const Column& c = b.columns[col];
      int64_t first = c.offset / 8, last = (c.offset + c.length + 7) / 8;
      if (last > first) EF_CUDA(cudaMemcpyAsync(bits.get() + pos, c.values + first, (size_t)(last - first), from, s));
      pos += last - first;
    }
    if (seg.empty()) seg.push_back({0, -1, 0, 0});
    DeviceBuffer<Segment> dseg(seg.size(), s);
    EF_CUDA(cudaMemcpyAsync(dseg.get(), seg.data(), seg.size() * sizeof(Segment), cudaMemcpyHostToDevice, s));
    if (d.rows) expand_validity<<<blocks_for(d.rows, 256), 256, 0, s>>>(bits.get(), dseg.get(), (int)seg.size(), d.rows, d.data.get());
    EF_CUDA(cudaStreamSynchronize(s));
  } else if (d.kind != Kind::Null) {
    d.width = fixed_width(r.fields[col].format);
    if (!d.width) fail(EINFOLD_INVALID, "a column of an unsupported type");
    if (r.device >= 0 && r.batches.size() == 1) {
      // One batch already in HBM: read in place.
      const Column& c = r.batches[0].columns[col];
      d.alias = c.values + c.offset * d.width;
    } else {
      d.data.allocate((size_t)(d.rows * d.width ? d.rows * d.width : 1), s);
      int64_t row = 0;
      for (auto& b : r.batches) {
        const Column& c = b.columns[col];
        if (c.length)
          EF_CUDA(cudaMemcpyAsync(d.data.get() + row * d.width, c.values + c.offset * d.width,
                                  (size_t)(c.length * d.width), from, s));
        row += c.length;
      }
    }
  }
  if (with_validity && d.nulls > 0) {
    d.valid.allocate((size_t)d.rows, s);
    std::vector<Segment> seg;
    int64_t nbytes = 0, row = 0;
    for (auto& b : r.batches) {
      const Column& c = b.columns[col];
      if (c.validity && c.nulls() > 0) {
        int64_t first = c.offset / 8, last = (c.offset + c.length + 7) / 8;
        seg.push_back({row, nbytes, (int32_t)(c.offset % 8), 0});
        nbytes += last - first;
      } else {
        seg.push_back({row, -1, 0, 0});
      }
      row += c.length;
    }
    DeviceBuffer<uint8_t> bits((size_t)(nbytes ? nbytes : 1), s);
    int64_t pos = 0;
    for (auto& b : r.batches) {
      const Column& c = b.columns[col];
      if (c.validity && c.nulls() > 0) {
        int64_t first = c.offset / 8, last = (c.offset + c.length + 7) / 8;
        EF_CUDA(cudaMemcpyAsync(bits.get() + pos, c.validity + first, (size_t)(last - first), from, s));
        pos += last - first;
      }
    }
    DeviceBuffer<Segment> dseg(seg.size(), s);
    EF_CUDA(cudaMemcpyAsync(dseg.get(), seg.data(), seg.size() * sizeof(Segment), cudaMemcpyHostToDevice, s));
    expand_validity<<<blocks_for(d.rows, 256), 256, 0, s>>>(bits.get(), dseg.get(), (int)seg.size(), d.rows, d.valid.get());
    EF_LAUNCH_CHECK();
    ctx.kernels++;
    EF_CUDA(cudaStreamSynchronize(s));  // `seg` is a host temporary
  }
  return d;
}

DeviceBuffer<int64_t> keys_as_i64(Context& ctx, const DeviceColumn& c, KeyStats* stats) {
  cudaStream_t s = ctx.stream;
  DeviceBuffer<int64_t> out((size_t)(c.rows ? c.rows : 1), s);
  DeviceBuffer<unsigned long long> mx(1, s);
  DeviceBuffer<int> flags(1, s);
  mx.zero();
  flags.zero();
  unsigned g = blocks_for(c.rows, 256);
  switch (c.kind) {
    case Kind::Int8: widen<int8_t><<<g, 256, 0, s>>>((const int8_t*)c.ptr(), c.rows, out.get(), mx.get(), flags.get()); break;
    case Kind::UInt8: widen<uint8_t><<<g, 256, 0, s>>>((const uint8_t*)c.ptr(), c.rows, out.get(), mx.get(), flags.get()); break;
    case Kind::Int16: widen<int16_t><<<g, 256, 0, s>>>((const int16_t*)c.ptr(), c.rows, out.get(), mx.get(), flags.get()); break;
    case Kind::UInt16: widen<uint16_t><<<g, 256, 0, s>>>((const uint16_t*)c.ptr(), c.rows, out.get(), mx.get(), flags.get()); break;
    case Kind::Int32: widen<int32_t><<<g, 256, 0, s>>>((const int32_t*)c.ptr(), c.rows, out.get(), mx.get(), flags.get()); break;
    case Kind::UInt32: widen<uint32_t><<<g, 256, 0, s>>>((const uint32_t*)c.ptr(), c.rows, out.get(), mx.get(), flags.get()); break;
    case Kind::Int64: widen<int64_t><<<g, 256, 0, s>>>((const int64_t*)c.ptr(), c.rows, out.get(), mx.get(), flags.get()); break;
    case Kind::UInt64: widen<uint64_t><<<g, 256, 0, s>>>((const uint64_t*)c.ptr(), c.rows, out.get(), mx.get(), flags.get()); break;
    default: fail(EINFOLD_INVALID, "keys_as_i64 of a non-integer column");
  }
  EF_LAUNCH_CHECK();
  ctx.kernels++;
  unsigned long long m = 0;
  int f = 0;
  EF_CUDA(cudaMemcpyAsync(&m, mx.get(), 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(&f, flags.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  stats->max = c.rows ? (int64_t)m : -1;
  stats->negative = f & 1;
  stats->too_large = (f & 2) != 0;
  return out;
}

void key_stats_i64(Context& ctx, const int64_t* keys, int64_t n, KeyStats* stats) {
  cudaStream_t s = ctx.stream;
  DeviceBuffer<unsigned long long> mx(1, s);
  DeviceBuffer<int> flags(1, s);
  mx.zero();
  flags.zero();
  widen<int64_t><<<blocks_for(n, 256), 256, 0, s>>>(keys, n, nullptr, mx.get(), flags.get());
  EF_LAUNCH_CHECK();
  ctx.kernels++;
  unsigned long long m = 0;
  int f = 0;
  EF_CUDA(cudaMemcpyAsync(&m, mx.get(), 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(&f, flags.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  stats->max = n ? (int64_t)m : -1;
  stats->negative = f & 1;
  stats->too_large = (f & 2) != 0;
}

int64_t exclusive_scan_flags(Context& ctx, const uint8_t* flags, int64_t n, int64_t* out) {
  cudaStream_t s = ctx.stream;
  if (n <= 0) return 0;
  size_t temp = 0;
  cub::TransformInputIterator<int64_t, cub::CastOp<int64_t>, const uint8_t*> it(flags, cub::CastOp<int64_t>());
  EF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, it, out, n, s));
  DeviceBuffer<uint8_t> t(temp ? temp : 1, s);
  EF_CUDA(cub::DeviceScan::ExclusiveSum(t.get(), temp, it, out, n, s));
  int64_t last = 0;
  uint8_t lastf = 0;
  EF_CUDA(cudaMemcpyAsync(&last, out + n - 1, 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(&lastf, flags + n - 1, 1, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  ctx.kernels += 2;
  return last + (lastf ? 1 : 0);
}

void pack_bits(Context& ctx, const uint8_t* bytes, int64_t n, uint8_t* bits) {
  if (n <= 0) return;
  pack_bits_kernel<<<blocks_for((n + 7) / 8, 256), 256, 0, ctx.stream>>>(bytes, n, bits);
  EF_LAUNCH_CHECK();
  ctx.kernels++;
}

HostBuffer to_host(Context& ctx, const void* dev, size_t bytes) {
  HostBuffer h = HostBuffer::page_locked(bytes ? bytes : 1);
  if (bytes) {
    EF_CUDA(cudaMemcpyAsync(h.ptr, dev, bytes, cudaMemcpyDeviceToHost, ctx.stream));
    EF_CUDA(cudaStreamSynchronize(ctx.stream));
  }
  h.bytes = bytes;
  return h;
}

__global__ void key_tables(int64_t n, OutKeys keys, int in_x, int64_t* __restrict__ tables) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < keys.n; k++)
      if (keys.key[k].in_x == in_x) tables[(int64_t)k * n + p] = keys.key[k].at(p, p);
}

StagedKeys stage_keys(Context& ctx, const OperandD& op, const Relation& r) {
  StagedKeys s;
  for (auto& k : op.keys) {
    const Field& f = r.fields[k.col];
    if (f.dictionary || !is_integer(f.kind)) decline("a key column that isn't integers");
    for (auto& b : r.batches)
      if (b.columns[k.col].nulls() > 0) decline("a NULL key");
    s.cols.push_back(stage_column(ctx, r, k.col, false));
    DeviceColumn& c = s.cols.back();
    KeyStats st;
    if (c.kind == Kind::Int64) {
      key_stats_i64(ctx, (const int64_t*)c.ptr(), c.rows, &st);
      s.keys.push_back((const int64_t*)c.ptr());
    } else {
      s.wide.push_back(keys_as_i64(ctx, c, &st));
      s.keys.push_back(s.wide.back().get());
    }
    if (st.negative || st.too_large) decline("a negative key, or one too large for int64");
    if (st.max == INT64_MAX) decline("a key whose extent doesn't fit");
    s.extent.push_back(st.max + 1);
  }
  return s;
}

Role role_of(const std::vector<int>& dims, const OperandD& op, const StagedKeys& s, const std::vector<int64_t>& extent) {
  Role r;
  if (dims.size() > (size_t)kMaxDims) decline("more than 8 dimensions in one role");
  for (int d : dims) {
    int slot = -1;
    for (size_t i = 0; i < op.keys.size(); i++)
      if (op.keys[i].dim == d) slot = (int)i;
    r.keys[r.n] = s.keys[slot];
    r.extent[r.n] = extent[d];
    r.n++;
  }
  return r;
}

}  // namespace ef
