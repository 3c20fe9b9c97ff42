// The dense fold on the device (crates/einfold-kernels/src/dense.rs:176-578).
//
// Host side: the reference's control logic, dimension roles W/X/Z/Y, the
// decline rules, the budget. Device side: every pass over rows or cells:
// keys to int64 with their extents, positions, the scatter of both operands
// into dense matrices with duplicate detection (integer atomics on flags
// only), the product, each domain row's cell, and the output's columns.
//
// Layout in HBM: a[x][z] (z contiguous: the product's K-major A), held[x][z]
// as int32 (0 absent, 1 NULL, 2 valued), b transposed as bt[w][y][z] (each
// column of b contiguous: the product's K-major B), reached[x] and valued[x]
// as bytes, and the product out[x][y].
#include <cmath>

#include "fold.h"
#include "gemm.cuh"
#include "stage.cuh"

namespace ef {
namespace {

enum : unsigned { F_DUP_A = 1, F_DUP_B = 2, F_NONFINITE_A = 4, F_NONFINITE_B = 8, F_REPEATED = 16 };
constexpr int64_t kFewCells = 4096;
constexpr int64_t kZBlock = 4096;
constexpr int64_t kNoGroup = -1;

// Scatters a's rows into a[x][z]; `held` packs a 2-bit code per cell (0
// absent, 1 NULL factor, 2 valued), 16 cells a word, so that a repeated
// position shows in the bits an atomic OR returns. The lanes of a warp that
// share a word OR their codes together first and one of them issues the
// atomic (rows in key order share words). Every thread of a block runs the same iterations,
// so the warp-wide matches see all the warp's rows. NARROW: word indices fit 32 bits.
template <bool NARROW>
__global__ void scatter_a_kernel(Role xs, Role zs, int64_t rows, const double* __restrict__ vals,
                                 const uint8_t* __restrict__ valid, int64_t nz, double* __restrict__ a,
                                 uint32_t* __restrict__ held, uint8_t* __restrict__ reached,
                                 uint8_t* __restrict__ valued, unsigned* flags) {
  unsigned f = 0;
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < rows; base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = base + threadIdx.x;
    const unsigned active = __ballot_sync(0xffffffffu, r < rows);
    if (r >= rows) continue;
    const int64_t x = role_position(xs, r), z = role_position(zs, r);
    const int64_t p = x * nz + z;
    const bool v = valid ? valid[r] != 0 : true;
    const unsigned sh = (unsigned)(p & 15) * 2;
    const unsigned long long word = (unsigned long long)(p >> 4);
    const unsigned same_word = NARROW ? __match_any_sync(active, (unsigned)word) : __match_any_sync(active, word);
    const unsigned bits = __reduce_or_sync(same_word, (v ? 2u : 1u) << sh);
    // A cell twice in the warp leaves fewer distinct cells than lanes.
    if (__popc(__reduce_or_sync(same_word, 1u << (p & 15))) != __popc(same_word)) f |= F_DUP_A;
    const int leader = __ffs(same_word) - 1;
    unsigned old = 0;
    if (lane == leader) old = atomicOr(&held[word], bits);
    old = __shfl_sync(same_word, old, leader);
    if ((old >> sh) & 3u) f |= F_DUP_A;
    reached[x] = 1;
    if (v) {
      const double val = vals[r];
      a[p] = val;
      valued[x] = 1;
      if (!isfinite(val)) f |= F_NONFINITE_A;
    }
  }
  if (f) atomicOr(flags, f);
}

// Scatters b's rows into b[w][z][y] (its natural layout: each row of b's
// matrix contiguous); `present` packs a bit per cell, ORed per word across
// the warp's lanes first as in scatter_a_kernel.
template <bool NARROW>
__global__ void scatter_b_kernel(Role wzs, Role ys, int64_t rows, const double* __restrict__ vals,
                                 const uint8_t* __restrict__ valid, int64_t ny, double* __restrict__ bm,
                                 uint32_t* __restrict__ present, unsigned* flags) {
  unsigned f = 0;
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < rows; base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = base + threadIdx.x;
    const unsigned active = __ballot_sync(0xffffffffu, r < rows);
    if (r >= rows) continue;
    const int64_t p = role_position(wzs, r) * ny + role_position(ys, r);
    const unsigned bit = 1u << (p & 31);
    const unsigned long long word = (unsigned long long)(p >> 5);
    const unsigned same_word = NARROW ? __match_any_sync(active, (unsigned)word) : __match_any_sync(active, word);
    const unsigned bits = __reduce_or_sync(same_word, bit);
    // A cell twice in the warp leaves fewer distinct bits than lanes.
    if (__popc(bits) != __popc(same_word)) f |= F_DUP_B;
    const int leader = __ffs(same_word) - 1;
    unsigned old = 0;
    if (lane == leader) old = atomicOr(&present[word], bits);
    old = __shfl_sync(same_word, old, leader);
    if (old & bit) f |= F_DUP_B;
    if (!valid || valid[r]) {
      const double val = vals[r];
      bm[p] = val;
      if (!isfinite(val)) f |= F_NONFINITE_B;
    }
  }
  if (f) atomicOr(flags, f);
}

struct Conds {
  int n = 0;
  KeyAt left[kMaxDims], right[kMaxDims];
  int cmp[kMaxDims];
  int64_t offset[kMaxDims];
  __device__ bool allowed(int64_t x, int64_t y) const {
    for (int i = 0; i < n; i++) {
      const __int128 l = left[i].at(x, y), r = (__int128)right[i].at(x, y) + offset[i];
      bool ok;
      switch (cmp[i]) {
        case 0: ok = l < r; break;
        case 1: ok = l <= r; break;
        case 2: ok = l > r; break;
        default: ok = l >= r; break;
      }
      if (!ok) return false;
    }
    return true;
  }
};

// Which cells are output rows: reached x and, with conditions, allowed (x, y).
__global__ void select_cells(int64_t nx, int64_t ny, const uint8_t* __restrict__ reached, Conds c,
                             uint8_t* __restrict__ sel) {
  for (int64_t x = blockIdx.y; x < nx; x += gridDim.y) {
    const bool r = reached[x] != 0;
    for (int64_t y = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; y < ny; y += (int64_t)gridDim.x * blockDim.x)
      sel[x * ny + y] = r && c.allowed(x, y);
  }
}

// Writes the output rows: cell (x, y) goes to pos[x*ny + y] when `sel` is
// given (conditions), else to row_index[x]·ny + y for reached x.
__global__ void emit_cells(int64_t nx, int64_t ny, const uint8_t* __restrict__ reached,
                           const int64_t* __restrict__ row_index, const uint8_t* __restrict__ sel,
                           const int64_t* __restrict__ pos, OutKeys keys, const int64_t* __restrict__ xtab,
                           const int64_t* __restrict__ ytab, const double* __restrict__ out,
                           const uint8_t* __restrict__ valued, double* __restrict__ val_out,
                           uint8_t* __restrict__ valid_out, unsigned long long* nulls) {
  unsigned long long local = 0;
  for (int64_t x = blockIdx.y; x < nx; x += gridDim.y) {
    if (!reached[x]) continue;
    const uint8_t v = valued[x];
    const int64_t base = sel ? 0 : row_index[x] * ny;
    for (int64_t y = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; y < ny; y += (int64_t)gridDim.x * blockDim.x) {
      const int64_t i = x * ny + y;
      if (sel && !sel[i]) continue;
      const int64_t o = sel ? pos[i] : base + y;
      for (int k = 0; k < keys.n; k++)
        store_key(keys.out[k], keys.width[k], o, keys.key[k].in_x ? xtab[(int64_t)k * nx + x] : ytab[(int64_t)k * ny + y]);
      val_out[o] = out[i];
      valid_out[o] = v;
      local += !v;
    }
  }
  if (local) atomicAdd(nulls, local);
}

// emit_cells for the common case, no conditions, keys of 8 bytes and an
// even ny: two cells a thread, each column written 16 bytes at a time.
__global__ void emit_cell_pairs(int64_t nx, int64_t ny, const uint8_t* __restrict__ reached,
                                const int64_t* __restrict__ row_index, OutKeys keys,
                                const int64_t* __restrict__ xtab, const int64_t* __restrict__ ytab,
                                const double* __restrict__ out, const uint8_t* __restrict__ valued,
                                double* __restrict__ val_out, uint8_t* __restrict__ valid_out,
                                unsigned long long* nulls) {
  unsigned long long local = 0;
  for (int64_t x = blockIdx.y; x < nx; x += gridDim.y) {
    if (!reached[x]) continue;
    const uint8_t v = valued[x];
    const int64_t base = row_index[x] * ny;
    for (int64_t y = 2 * ((int64_t)blockIdx.x * blockDim.x + threadIdx.x); y < ny;
         y += 2 * (int64_t)gridDim.x * blockDim.x) {
      const int64_t o = base + y, i = x * ny + y;
      for (int k = 0; k < keys.n; k++) {
        longlong2 kv;
        if (keys.key[k].in_x) {
          kv.x = kv.y = xtab[(int64_t)k * nx + x];
        } else {
          kv = *(const longlong2*)(ytab + (int64_t)k * ny + y);
        }
        *(longlong2*)((int64_t*)keys.out[k] + o) = kv;
      }
      *(double2*)(val_out + o) = *(const double2*)(out + i);
      *(uchar2*)(valid_out + o) = make_uchar2(v, v);
      local += v ? 0 : 2;
    }
  }
  if (local) atomicAdd(nulls, local);
}

struct DomainKeys {
  int n = 0;
  const int64_t* key[kMaxDims];
  const uint8_t* valid[kMaxDims];
  int64_t extent[kMaxDims], stride[kMaxDims];
};

__global__ void locate_kernel(DomainKeys k, int64_t rows, int64_t* __restrict__ cell) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = 0;
    for (int i = 0; i < k.n && c != kNoGroup; i++) {
      const int64_t v = k.key[i][r];
      const bool ok = (!k.valid[i] || k.valid[i][r]) && v >= 0 && v < k.extent[i];
      c = ok ? c + v * k.stride[i] : kNoGroup;
    }
    cell[r] = c;
  }
}

__global__ void unique_cells(int64_t rows, const int64_t* __restrict__ cell, int32_t* __restrict__ seen,
                             unsigned* flags) {
  unsigned f = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = cell[r];
    if (c != kNoGroup && atomicExch(&seen[c], 1) != 0) f |= F_REPEATED;
  }
  if (f) atomicOr(flags, f);
}

__global__ void domain_values(int64_t rows, const int64_t* __restrict__ cell, int64_t ny,
                              const uint8_t* __restrict__ valued, Conds c, const double* __restrict__ out,
                              int has_missing, double missing, double* __restrict__ val, uint8_t* __restrict__ valid) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t cl = cell[r];
    bool has = cl != kNoGroup;
    if (has) {
      const int64_t x = cl / ny, y = cl % ny;
      if (c.n && !c.allowed(x, y)) has = false;
      else if (valued && !valued[x]) has = false;
    }
    if (has) {
      val[r] = out[cl];
      valid[r] = 1;
    } else {
      val[r] = has_missing ? missing : 0.0;
      valid[r] = (uint8_t)(has_missing ? 1 : 0);
    }
  }
}

bool worth(uint64_t cells, uint64_t rows) {
  return cells <= sat_add(sat_mul(rows, 4), (uint64_t)kFewCells) && cells < UINT32_MAX;
}

}  // namespace

FoldOutput dense_fold(Context& ctx, const FoldD& f, const Relation& a, const Relation& b, const Relation* domain,
                      const std::vector<Field>& schema, const einfold_options& o, Budget& budget) {
  cudaStream_t s = ctx.stream;
  if (f.operands.size() != 2) decline("not two operands");
  const OperandD& op_a = f.operands[0];
  const OperandD& op_b = f.operands[1];
  if (f.row_expr) decline("a row expression");
  // Roles (dense.rs:196-219): W, X, Y in output order, Z in dimension order.
  std::vector<int> ws, xs, ys, zs;
  for (auto& out : f.outputs) {
    bool ha = op_a.holds(out.dim), hb = op_b.holds(out.dim);
    if (ha && hb) ws.push_back(out.dim);
    else if (ha) xs.push_back(out.dim);
    else if (hb) ys.push_back(out.dim);
    else decline("an output neither operand holds");
  }
  xs.insert(xs.begin(), ws.begin(), ws.end());
  for (int d = 0; d < f.n_dims(); d++)
    if (f.is_aggregated(d)) {
      if (!op_a.holds(d) || !op_b.holds(d)) decline("a summed dimension one operand lacks");
      zs.push_back(d);
    }
  auto is_output = [&](int d) {
    for (int x : xs) if (x == d) return true;
    for (int y : ys) if (y == d) return true;
    return false;
  };
  for (auto& c : f.conditions)
    if (!is_output(c.left) || !is_output(c.right)) decline("a condition on a summed dimension");
  auto integers = [&](const OperandD& op, const Relation& r) {
    if (r.batches.empty()) return true;
    for (auto& k : op.keys) {
      const Field& fl = r.fields[k.col];
      if (fl.dictionary || !is_integer(fl.kind)) return false;
    }
    return true;
  };
  if (!integers(op_a, a) || !integers(op_b, b)) decline("keys that aren't integers");
  const uint64_t ra = (uint64_t)a.rows(), rb = (uint64_t)b.rows();
  budget.reserve(sat_mul(sat_add(sat_mul(ra, op_a.keys.size()), sat_mul(rb, op_b.keys.size())), 8),
                 "the dense algorithm's keys");
  ctx.phase("dense: checks");
  StagedKeys ka = stage_keys(ctx, op_a, a), kb = stage_keys(ctx, op_b, b);
  ctx.phase("dense: keys");
  std::vector<int64_t> extent(f.n_dims(), 0);
  for (size_t i = 0; i < op_a.keys.size(); i++) extent[op_a.keys[i].dim] = std::max(extent[op_a.keys[i].dim], ka.extent[i]);
  for (size_t i = 0; i < op_b.keys.size(); i++) extent[op_b.keys[i].dim] = std::max(extent[op_b.keys[i].dim], kb.extent[i]);
  auto size = [&](const std::vector<int>& dims, uint64_t* out) {
    uint64_t n = 1;
    for (int d : dims)
      if (!checked_mul(n, (uint64_t)extent[d], &n)) return false;
    *out = n;
    return true;
  };
  std::vector<int> wzs = ws;
  wzs.insert(wzs.end(), zs.begin(), zs.end());
  uint64_t nw, nx, nz, ny;
  if (!size(ws, &nw) || !size(xs, &nx) || !size(zs, &nz) || !size(ys, &ny)) decline("sizes that overflow");
  const uint64_t per_batch = nw ? nx / nw : 0;
  const uint64_t out_rows = domain ? (uint64_t)domain->rows() : sat_mul(nx, ny);
  if (!worth(sat_mul(nx, nz), ra) || !worth(sat_mul(sat_mul(nw, nz), ny), rb) || !worth(sat_mul(nx, ny), out_rows))
    decline("too sparse for dense matrices");
  const uint64_t na = nx * nz, nb = nw * nz * ny;
  const uint64_t out_columns = f.outputs.size() + 1 + (domain ? 1 : 0);
  const uint64_t working = sat_add(sat_add(sat_add(sat_mul(na, 12), sat_mul(nx, 2)), sat_add(sat_mul(nb, 12), sat_mul(ra + rb, 8))),
                                   sat_add(sat_mul(sat_mul(nx, ny), 16), sat_mul(sat_mul(out_rows, out_columns), 8)));
  budget.reserve(working, "the dense algorithm's matrices");
  const bool zero_default = f.domain && f.domain->has_missing && std::signbit(f.domain->missing) == false &&
                            f.domain->missing == 0.0;

  // The operands' factors.
  if (op_a.factor < 0 || op_b.factor < 0) decline("an operand without a factor");
  if (a.fields[op_a.factor].kind != Kind::Float64 || a.fields[op_a.factor].dictionary) decline("factors that aren't Float64");
  if (b.fields[op_b.factor].kind != Kind::Float64 || b.fields[op_b.factor].dictionary) decline("factors that aren't Float64");
  DeviceColumn fa = stage_column(ctx, a, op_a.factor), fb = stage_column(ctx, b, op_b.factor);
  ctx.phase("dense: factors staged");

  DeviceBuffer<double> am(na, s), bm(nb, s), out(nx * ny, s);
  DeviceBuffer<uint32_t> held((na + 15) / 16, s), present((nb + 31) / 32, s);
  DeviceBuffer<uint8_t> reached(nx, s), valued(nx, s);
  DeviceBuffer<unsigned> flags(1, s);
  ctx.phase("dense: matrices reserved");
  // Cells no row writes must read as 0: only incomplete operands or NULL
  // factors leave any (a repeated row declines below).
  if (ra < na || fa.nulls > 0) am.zero();
  if (rb < nb || fb.nulls > 0) bm.zero();
  held.zero(); present.zero(); reached.zero(); valued.zero(); flags.zero();
  ctx.phase("dense: matrices allocated");
  Role rxs = role_of(xs, op_a, ka, extent), rzs = role_of(zs, op_a, ka, extent);
  Role rwzs = role_of(wzs, op_b, kb, extent), rys = role_of(ys, op_b, kb, extent);
  if (ra) {
    auto scatter_a = na / 16 < (1ull << 32) ? scatter_a_kernel<true> : scatter_a_kernel<false>;
    scatter_a<<<blocks_for(ra, 256), 256, 0, s>>>(rxs, rzs, (int64_t)ra, (const double*)fa.ptr(), fa.valid.get(),
                                                  (int64_t)nz, am.get(), held.get(), reached.get(), valued.get(),
                                                  flags.get());
    ctx.kernels++;
  }
  if (rb) {
    auto scatter_b = nb / 32 < (1ull << 32) ? scatter_b_kernel<true> : scatter_b_kernel<false>;
    scatter_b<<<blocks_for(rb, 256), 256, 0, s>>>(rwzs, rys, (int64_t)rb, (const double*)fb.ptr(), fb.valid.get(),
                                                  (int64_t)ny, bm.get(), present.get(), flags.get());
    ctx.kernels++;
  }
  EF_LAUNCH_CHECK();
  ctx.phase("dense: scatter");
  unsigned fl = 0;
  EF_CUDA(cudaMemcpyAsync(&fl, flags.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  if (fl & F_DUP_A) decline("duplicate key tuples in a");
  if (fl & F_DUP_B) decline("duplicate key tuples in b");
  const bool finite = !(fl & F_NONFINITE_A);
  // Without duplicates, every row of b holds its own cell.
  const bool holes = fb.nulls > 0 || rb < nb;
  if (holes && (!zero_default || !finite)) decline("holes in b without a 0.0 default over finite factors");
  present.reset();

  // The fold's conditions, on output keys.
  std::vector<int> order = xs;
  order.insert(order.end(), ys.begin(), ys.end());
  auto key_at = [&](int d) {
    KeyAt k{};
    bool in_x = false;
    for (int x : xs) in_x |= x == d;
    const std::vector<int>& role = in_x ? xs : ys;
    size_t slot = 0;
    while (role[slot] != d) slot++;
    int64_t stride = 1;
    for (size_t i = slot + 1; i < role.size(); i++) stride *= extent[role[i]];
    k.in_x = in_x;
    k.stride = stride;
    k.extent = extent[d] ? extent[d] : 1;
    return k;
  };
  Conds conds;
  if (f.conditions.size() > (size_t)kMaxDims) decline("more than 8 conditions");
  for (auto& c : f.conditions) {
    conds.left[conds.n] = key_at(c.left);
    conds.right[conds.n] = key_at(c.right);
    conds.cmp[conds.n] = c.cmp;
    conds.offset[conds.n] = c.offset;
    conds.n++;
  }

  // Each domain row's cell, before the product (dense.rs:400-434).
  DeviceBuffer<int64_t> cells;
  int64_t nd = 0;
  if (f.domain && domain) {
    nd = domain->rows();
    cells.allocate((size_t)(nd ? nd : 1), s);
    DomainKeys dk;
    std::vector<DeviceColumn> dcols;
    std::vector<DeviceBuffer<int64_t>> dkeys;
    if (f.outputs.size() > (size_t)kMaxDims) decline("more than 8 outputs");
    for (auto& out_d : f.outputs) {
      dcols.push_back(stage_column(ctx, *domain, out_d.domain_col, true));
      DeviceColumn& c = dcols.back();
      if (!is_integer(c.kind)) fail(EINFOLD_INVALID, "a domain key column that isn't integers");
      KeyStats st;
      dkeys.push_back(keys_as_i64(ctx, c, &st));
      int64_t stride = 1;
      size_t slot = 0;
      while (order[slot] != out_d.dim) slot++;
      for (size_t i = slot + 1; i < order.size(); i++) stride *= extent[order[i]];
      dk.key[dk.n] = dkeys.back().get();
      dk.valid[dk.n] = c.valid.get();
      dk.extent[dk.n] = extent[out_d.dim];
      dk.stride[dk.n] = stride;
      dk.n++;
    }
    if (nd) {
      locate_kernel<<<blocks_for(nd, 256), 256, 0, s>>>(dk, nd, cells.get());
      ctx.kernels++;
    }
    if (o.domain_rows == 1 && nd) {
      DeviceBuffer<int32_t> seen(nx * ny, s);
      seen.zero();
      unique_cells<<<blocks_for(nd, 256), 256, 0, s>>>(nd, cells.get(), seen.get(), flags.get());
      ctx.kernels++;
      EF_LAUNCH_CHECK();
      EF_CUDA(cudaMemcpyAsync(&fl, flags.get(), 4, cudaMemcpyDeviceToHost, s));
      EF_CUDA(cudaStreamSynchronize(s));
      if (fl & F_REPEATED) decline("two domain rows with one cell");
    }
  }

  // The product (dense.rs:442-467 and accumulate, :706-770).
  const bool split = o.precision == 0 && finite && !(fl & F_NONFINITE_B);
  if (nx && ny) {
    if (split) {
      split_gemm(ctx, am.get(), bm.get(), true, out.get(), (int64_t)nw, (int64_t)per_batch, (int64_t)ny,
                 (int64_t)nz, o.slices ? o.slices : kDefaultSlices, s);
    } else {
      fp64_gemm(ctx, am.get(), held.get(), bm.get(), out.get(), (int64_t)nw, (int64_t)per_batch, (int64_t)ny,
                (int64_t)nz, 0, (int64_t)(nx * ny >= (uint64_t)kFewCells ? 0 : kZBlock), false, s);
    }
  }
  ctx.phase("dense: product");
  am.reset();
  bm.reset();
  held.reset();

  FoldOutput result;
  result.algorithm = EINFOLD_ALG_DENSE;
  if (f.domain && domain) {
    if (o.result_on_device) fail(EINFOLD_INVALID, "results in device memory are not supported with a domain");
    const DomainD& spec = *f.domain;
    DeviceBuffer<double> val((size_t)(nd ? nd : 1), s);
    DeviceBuffer<uint8_t> valid((size_t)(nd ? nd : 1), s);
    if (nd) {
      domain_values<<<blocks_for(nd, 256), 256, 0, s>>>(nd, cells.get(), (int64_t)(ny ? ny : 1),
                                                        zero_default ? nullptr : valued.get(), conds, out.get(),
                                                        spec.has_missing, spec.missing, val.get(), valid.get());
      ctx.kernels++;
      EF_LAUNCH_CHECK();
    }
    HostBuffer hv = to_host(ctx, val.get(), (size_t)nd * 8);
    HostBuffer hvalid = to_host(ctx, valid.get(), (size_t)nd);
    int64_t off = 0;
    for (auto& batch : domain->batches) {
      OutBatch ob;
      ob.rows = batch.rows;
      for (size_t i = 0; i < spec.carry.size(); i++) {
        OutColumn c = copy_column(batch.columns[spec.carry[i]], domain->fields[spec.carry[i]]);
        c.format = schema[i].format;
        c.name = schema[i].name;
        ob.columns.push_back(std::move(c));
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
      ob.columns.push_back(std::move(v));
      result.batches.push_back(std::move(ob));
      off += batch.rows;
    }
    return result;
  }
  if (f.domain || domain) fail(EINFOLD_INVALID, "a fold with a domain was given no domain relation");

  // Output rows (dense.rs:516-575): (x, y) for each reached x, in order, every
  // y, minus the groups the conditions disallow.
  const int64_t cells_n = (int64_t)(nx * ny);
  OutKeys ok;
  if (f.outputs.size() > (size_t)kMaxDims) decline("more than 8 outputs");
  for (size_t i = 0; i < f.outputs.size(); i++) {
    ok.key[ok.n] = key_at(f.outputs[i].dim);
    ok.width[ok.n] = width_of(schema[i].kind);
    ok.n++;
  }
  DeviceBuffer<int64_t> xtab((size_t)(ok.n * nx ? ok.n * nx : 1), s), ytab((size_t)(ok.n * ny ? ok.n * ny : 1), s);
  if (nx) key_tables<<<blocks_for(nx, 256), 256, 0, s>>>((int64_t)nx, ok, 1, xtab.get());
  if (ny) key_tables<<<blocks_for(ny, 256), 256, 0, s>>>((int64_t)ny, ok, 0, ytab.get());
  ctx.kernels += 2;
  DeviceBuffer<uint8_t> sel;
  DeviceBuffer<int64_t> pos, row_index;
  // Blocks of 256 cells of a row, each block walking rows x, x + gridDim.y,
  // ... (about 16 blocks an SM).
  const uint64_t gx = std::min<uint64_t>(std::max<uint64_t>((ny + 255) / 256, 1), 64);
  const dim3 grid2((unsigned)gx, (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(nx, 148 * 16 / gx)));
  int64_t n_out;
  if (conds.n) {
    sel.allocate((size_t)(cells_n ? cells_n : 1), s);
    pos.allocate((size_t)(cells_n ? cells_n : 1), s);
    if (cells_n) {
      select_cells<<<grid2, 256, 0, s>>>((int64_t)nx, (int64_t)ny, reached.get(), conds, sel.get());
      ctx.kernels++;
      EF_LAUNCH_CHECK();
    }
    n_out = exclusive_scan_flags(ctx, sel.get(), cells_n, pos.get());
  } else {
    row_index.allocate((size_t)(nx ? nx : 1), s);
    n_out = exclusive_scan_flags(ctx, reached.get(), (int64_t)nx, row_index.get()) * (int64_t)ny;
  }
  ctx.phase("dense: select");
  std::vector<DeviceBuffer<uint8_t>> key_dev;
  for (int i = 0; i < ok.n; i++) {
    key_dev.emplace_back((size_t)(n_out ? n_out * ok.width[i] : 1), s);
    ok.out[i] = key_dev.back().get();
  }
  DeviceBuffer<double> vals((size_t)(n_out ? n_out : 1), s);
  DeviceBuffer<uint8_t> vvalid((size_t)(n_out ? n_out : 1), s);
  DeviceBuffer<unsigned long long> nulls(1, s);
  nulls.zero();
  ctx.phase("dense: result reserved");
  bool pairs = !sel.get() && ny % 2 == 0;
  for (int k = 0; k < ok.n; k++) pairs = pairs && ok.width[k] == 8;
  if (cells_n && n_out && pairs) {
    const uint64_t gx = std::min<uint64_t>(std::max<uint64_t>((ny / 2 + 255) / 256, 1), 64);
    const dim3 grid_pairs((unsigned)gx, (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(nx, 148 * 16 / gx)));
    emit_cell_pairs<<<grid_pairs, 256, 0, s>>>((int64_t)nx, (int64_t)ny, reached.get(), row_index.get(), ok,
                                               xtab.get(), ytab.get(), out.get(), valued.get(), vals.get(),
                                               vvalid.get(), nulls.get());
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  } else if (cells_n && n_out) {
    emit_cells<<<grid2, 256, 0, s>>>((int64_t)nx, (int64_t)ny, reached.get(), row_index.get(), sel.get(), pos.get(), ok,
                                     xtab.get(), ytab.get(), out.get(), valued.get(), vals.get(), vvalid.get(),
                                     nulls.get());
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  }
  unsigned long long n_nulls = 0;
  EF_CUDA(cudaMemcpyAsync(&n_nulls, nulls.get(), 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  ctx.phase("dense: cells emitted");
  OutBatch ob;
  ob.rows = n_out;
  for (size_t i = 0; i < f.outputs.size(); i++) {
    OutColumn c;
    c.format = schema[i].format;
    c.name = schema[i].name;
    c.kind = schema[i].kind;
    c.nullable = schema[i].nullable;
    c.length = n_out;
    c.values = result_buffer(ctx, key_dev[i], (size_t)(n_out * ok.width[i]), o.result_on_device);
    ob.columns.push_back(std::move(c));
  }
  OutColumn v;
  v.format = "g";
  v.kind = Kind::Float64;
  v.name = schema.back().name;
  v.length = n_out;
  v.values = result_buffer(ctx, vals, (size_t)n_out * 8, o.result_on_device);
  v.null_count = (int64_t)n_nulls;
  if (n_nulls) {
    DeviceBuffer<uint8_t> bits((size_t)((n_out + 7) / 8), s);
    pack_bits(ctx, vvalid.get(), n_out, bits.get());
    v.validity = result_buffer(ctx, bits, (size_t)((n_out + 7) / 8), o.result_on_device);
  }
  EF_CUDA(cudaStreamSynchronize(s));
  ob.columns.push_back(std::move(v));
  result.batches.push_back(std::move(ob));
  ctx.phase("dense: result");
  return result;
}

}  // namespace ef
