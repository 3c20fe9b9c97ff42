// Chains of three operands (crates/einfold-kernels/src/chain.rs:64-288): a
// SUM of the product of three operands' factors, computed as two dense folds
// in the cheaper order, the first one's result left in HBM and read by the
// second as a device relation.
//
// Host side: the reference's control logic — the overflow guard (every
// non-NULL factor finite, Π max|f|·rows ≤ 2^1000), the extents, the pair
// contracted first (the cheapest of those sharing a dimension, the first of
// equals), the two folds and their numbering, and the swap of operands when
// the dense fold declines. Device side: the factors' statistics, and the
// dense folds.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fold.h"
#include "stage.cuh"

namespace ef {
namespace {

constexpr double kLargestBound = 1.0715086071862673e301;  // 2^1000 (chain.rs LARGEST_BOUND)

// max |v| over the valid rows (as ordered bits) and whether one isn't finite.
__global__ void factor_stats(int64_t n, const double* __restrict__ v, const uint8_t* __restrict__ valid,
                             unsigned long long* largest, unsigned* bad) {
  double m = 0.0;
  bool b = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (valid && !valid[i]) continue;
    const double a = fabs(v[i]);
    if (!(a <= 1.7976931348623157e308)) b = true;
    else m = fmax(m, a);
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  b = __any_sync(0xffffffffu, b);
  if ((threadIdx.x & 31) == 0) {
    if (m > 0.0) atomicMax(largest, (unsigned long long)__double_as_longlong(m));
    if (b) atomicOr(bad, 1u);
  }
}

// guarded (chain.rs:161-183).
bool guarded(Context& ctx, const FoldD& f, const std::vector<const Relation*>& ops) {
  cudaStream_t s = ctx.stream;
  double bound = 1.0;
  for (size_t i = 0; i < 3; i++) {
    const Relation& r = *ops[i];
    const int c = f.operands[i].factor;
    if (c < 0) return false;
    const Field& fd = r.fields[c];
    if (fd.dictionary || fd.kind != Kind::Float64) return false;
    const int64_t rows = r.rows();
    double largest = 0.0;
    if (rows > 0) {
      DeviceColumn col = stage_column(ctx, r, c, true);
      DeviceBuffer<unsigned long long> mx(1, s);
      DeviceBuffer<unsigned> bad(1, s);
      mx.zero();
      bad.zero();
      factor_stats<<<blocks_for((uint64_t)rows, 256), 256, 0, s>>>(rows, (const double*)col.ptr(),
                                                                  col.nulls ? col.valid.get() : nullptr, mx.get(),
                                                                  bad.get());
      EF_LAUNCH_CHECK();
      ctx.kernels++;
      unsigned long long m = 0;
      unsigned b = 0;
      EF_CUDA(cudaMemcpyAsync(&m, mx.get(), 8, cudaMemcpyDeviceToHost, s));
      EF_CUDA(cudaMemcpyAsync(&b, bad.get(), 4, cudaMemcpyDeviceToHost, s));
      EF_CUDA(cudaStreamSynchronize(s));
      if (b) return false;
      std::memcpy(&largest, &m, 8);
    }
    bound *= largest * (double)rows;
  }
  return bound <= kLargestBound;
}

std::vector<int> dims_of(const OperandD& op) {
  std::vector<int> d;
  for (auto& k : op.keys) d.push_back(k.dim);
  std::sort(d.begin(), d.end());
  return d;
}

std::vector<int> union_of(const std::vector<int>& a, const std::vector<int>& b) {
  std::vector<int> u = a;
  u.insert(u.end(), b.begin(), b.end());
  std::sort(u.begin(), u.end());
  u.erase(std::unique(u.begin(), u.end()), u.end());
  return u;
}

int place_of(const std::vector<int>& local, int d) {
  return (int)(std::find(local.begin(), local.end(), d) - local.begin());
}

// The first fold's kept dimensions: the outputs and those `rest` joins on.
std::vector<int> kept_of(const FoldD& f, const std::vector<int>& pair, int rest) {
  std::vector<int> k;
  for (int d : pair)
    if (f.output_of(d) >= 0 || f.operands[rest].holds(d)) k.push_back(d);
  return k;
}

OperandD renumbered(const OperandD& op, const std::vector<int>& local) {
  OperandD r;
  for (auto& k : op.keys) r.keys.push_back({place_of(local, k.dim), k.col});
  r.factor = op.factor;
  return r;
}

FoldD two_operand_fold(const FoldD& f, const std::vector<int>& local, OperandD a, OperandD b,
                       const std::vector<int>& outputs) {
  FoldD g;
  for (int d : local) g.equality.push_back(f.equality[d]);
  g.operands = {std::move(a), std::move(b)};
  for (int d : outputs) g.outputs.push_back(OutputD{place_of(local, d), -1, 0});
  return g;
}

// `fold` of a and b by the dense algorithm, or where it declines, of b and a
// (chain.rs:124-148).
FoldOutput either(Context& ctx, const FoldD& g, const Relation& a, const Relation& b,
                  const std::vector<Field>& schema, const einfold_options& o, Budget& budget) {
  try {
    return dense_fold(ctx, g, a, b, nullptr, schema, o, budget);
  } catch (const Declined&) {
  }
  FoldD swapped = g;
  std::swap(swapped.operands[0], swapped.operands[1]);
  return dense_fold(ctx, swapped, b, a, nullptr, schema, o, budget);
}

// A fold's device result as a relation the next fold reads in place.
Relation as_relation(const std::vector<OutBatch>& batches, const std::vector<Field>& schema, int device) {
  Relation r;
  r.fields = schema;
  r.device = device;
  for (auto& ob : batches) {
    Batch b;
    b.rows = ob.rows;
    for (auto& oc : ob.columns) {
      Column c;
      c.kind = oc.kind;
      c.length = oc.length;
      c.null_count = oc.null_count;
      c.validity = oc.null_count ? (const uint8_t*)oc.validity.ptr : nullptr;
      c.values = (const uint8_t*)oc.values.ptr;
      c.data = (const uint8_t*)oc.data.ptr;
      c.device = true;
      b.columns.push_back(c);
    }
    r.batches.push_back(std::move(b));
  }
  return r;
}

}  // namespace

FoldOutput chain_fold(Context& ctx, const FoldD& f, const std::vector<const Relation*>& ops,
                      const std::vector<Field>& schema, const einfold_options& o, Budget& budget) {
  bool chained = f.operands.size() == 3 && !f.row_expr && !f.domain && f.conditions.empty();
  for (auto& op : f.operands) chained = chained && op.factor >= 0;
  if (!chained) decline("not a chain of three products");
  if (!guarded(ctx, f, ops)) decline("a factor that isn't finite, or sums that could overflow");
  // Extents (chain.rs:188-200): the dense keys of every operand.
  std::vector<int64_t> extent((size_t)f.n_dims(), 0);
  for (size_t i = 0; i < 3; i++) {
    StagedKeys sk = stage_keys(ctx, f.operands[i], *ops[i]);
    for (size_t k = 0; k < f.operands[i].keys.size(); k++)
      extent[f.operands[i].keys[k].dim] = std::max(extent[f.operands[i].keys[k].dim], sk.extent[k]);
  }
  // The pair contracted first: the cheapest of those sharing a dimension.
  using u128 = unsigned __int128;
  auto product = [&](const std::vector<int>& dims, u128* out) {
    u128 n = 1;
    for (int d : dims) {
      const u128 e = (u128)(uint64_t)extent[d];
      if (e && n > ~(u128)0 / e) return false;
      n *= e;
    }
    *out = n;
    return true;
  };
  const int pairs[3][3] = {{0, 1, 2}, {1, 2, 0}, {0, 2, 1}};
  int best = -1;
  u128 best_cost = 0;
  for (int c = 0; c < 3; c++) {
    const int x = pairs[c][0], y = pairs[c][1], rest = pairs[c][2];
    const std::vector<int> dx = dims_of(f.operands[x]), dy = dims_of(f.operands[y]);
    bool shares = false;
    for (int d : dx) shares |= std::find(dy.begin(), dy.end(), d) != dy.end();
    if (!shares) continue;
    const std::vector<int> pair = union_of(dx, dy);
    const std::vector<int> second = union_of(kept_of(f, pair, rest), dims_of(f.operands[rest]));
    u128 a, b;
    if (!product(pair, &a) || !product(second, &b) || a > ~(u128)0 - b) continue;
    if (best < 0 || a + b < best_cost) {
      best = c;
      best_cost = a + b;
    }
  }
  if (best < 0) decline("no two operands share a dimension");
  const int x = pairs[best][0], y = pairs[best][1], rest = pairs[best][2];
  // The two folds (chain.rs:232-288), each numbering its own dimensions.
  const std::vector<int> pair = union_of(dims_of(f.operands[x]), dims_of(f.operands[y]));
  const std::vector<int> kept = kept_of(f, pair, rest);
  const FoldD first =
      two_operand_fold(f, pair, renumbered(f.operands[x], pair), renumbered(f.operands[y], pair), kept);
  const std::vector<int> local = union_of(kept, dims_of(f.operands[rest]));
  OperandD t;
  for (size_t c = 0; c < kept.size(); c++) t.keys.push_back({place_of(local, kept[c]), (int)c});
  t.factor = (int)kept.size();
  std::vector<int> outs;
  for (auto& out : f.outputs) outs.push_back(out.dim);
  const FoldD second = two_operand_fold(f, local, t, renumbered(f.operands[rest], local), outs);
  const std::vector<Field> first_schema = fold_schema(first, {&ops[x]->fields, &ops[y]->fields}, nullptr);
  einfold_options in_hbm = o;
  in_hbm.result_on_device = 1;
  FoldOutput tmp = either(ctx, first, *ops[x], *ops[y], first_schema, in_hbm, budget);
  ctx.phase("chain: first fold");
  const Relation t_rel = as_relation(tmp.batches, first_schema, ctx.device);
  FoldOutput out = either(ctx, second, t_rel, *ops[rest], schema, o, budget);
  ctx.phase("chain: second fold");
  return out;
}

}  // namespace ef
