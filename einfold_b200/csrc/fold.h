// The fold and pipeline descriptions, parsed from the C ABI's structs with
// the rules of crates/einfold-ir (Fold::try_new fold.rs:333-416,
// Fold::with_conditions, Pipeline::try_new pipeline.rs:216-300).
#pragma once

#include <optional>
#include <vector>

#include "arrow.h"
#include "common.h"

namespace ef {

struct KeyD {
  int dim, col;
};

struct OperandD {
  std::vector<KeyD> keys;
  int factor = -1;
  int column_of(int d) const {
    for (auto& k : keys)
      if (k.dim == d) return k.col;
    return -1;
  }
  bool holds(int d) const { return column_of(d) >= 0; }
};

struct OutputD {
  int dim = 0, domain_col = -1, domain_eq = 0;
};

struct ConditionD {
  int left = 0, cmp = 0, right = 0;
  int64_t offset = 0;
  // left <cmp> right + offset, in 128-bit integers (fold.rs:Condition::holds).
  bool holds(int64_t l, int64_t r) const {
    __int128 L = l, R = (__int128)r + offset;
    switch (cmp) {
      case 0: return L < R;
      case 1: return L <= R;
      case 2: return L > R;
      default: return L >= R;
    }
  }
  std::optional<ConditionD> mirrored() const {
    if (offset == INT64_MIN) return std::nullopt;
    static const int mirror[4] = {2, 3, 0, 1};
    return ConditionD{right, mirror[cmp], left, -offset};
  }
};

struct DomainD {
  std::vector<int> carry;
  bool has_missing = false;
  double missing = 0.0;
};

struct ExprNode {
  int kind = 0, a = 0, b = 0;
  double value = 0.0;
};

struct FoldD {
  std::vector<int> equality;
  std::vector<OperandD> operands;
  std::vector<OutputD> outputs;
  bool row_expr = false;
  std::vector<ExprNode> row;
  std::optional<DomainD> domain;
  std::vector<ConditionD> conditions;

  int n_dims() const { return (int)equality.size(); }
  int output_of(int d) const {
    for (size_t i = 0; i < outputs.size(); i++)
      if (outputs[i].dim == d) return (int)i;
    return -1;
  }
  bool is_aggregated(int d) const { return output_of(d) < 0; }
  // Columns an expression row reads, as (operand, column), in order.
  std::vector<std::pair<int, int>> row_columns() const {
    std::vector<std::pair<int, int>> out;
    for (auto& n : row)
      if (n.kind == 0) out.push_back({n.a, n.b});
    return out;
  }
};

FoldD parse_fold(const einfold_fold_desc* d);

struct PipelineD {
  FoldD producer;
  bool weight_expr = false;
  int scale_kind = 0;
  double scale_c = 1.0;
  int shift = 1;
  int normalizer = 0;
  std::vector<ExprNode> weight;
  std::vector<int> equality;  // own dimensions
  OperandD values;
  std::vector<int> outputs;
};

PipelineD parse_pipeline(const einfold_pipeline_desc* d);

// Output schema of a fold (schema.rs:40-143); `operands` are the operands'
// field lists, `domain` the domain's or null.
std::vector<Field> fold_schema(const FoldD& f, const std::vector<const std::vector<Field>*>& operands,
                               const std::vector<Field>* domain);
std::vector<Field> pipeline_schema(const PipelineD& p, const std::vector<const std::vector<Field>*>& inputs);

// Fold computations, each returning the result batches and, by pointer, the
// algorithm used; `Declined` is thrown where the reference returns None.
struct FoldOutput {
  std::vector<OutBatch> batches;
  int algorithm = EINFOLD_ALG_NONE;
  uint64_t tiles_visited = 0, tiles = 0;
};

FoldOutput dense_fold(Context& ctx, const FoldD& f, const Relation& a, const Relation& b, const Relation* domain,
                      const std::vector<Field>& schema, const einfold_options& o, Budget& budget);
// The ranks of the keys in columns `cols` of `r` (rank_columns,
// discriminate.rs:240-277): rank[i] per row, first[k] the smallest row of rank
// k; returns the number of ranks. Outputs in host memory, or device memory
// when `device_out`.
int64_t rank_columns(Context& ctx, const Relation& r, const std::vector<int>& cols, int float_keys, uint32_t* rank,
                     uint32_t* first, bool device_out);
FoldOutput discriminate_fold(Context& ctx, const FoldD& f, const Relation& a, const Relation& b,
                             const Relation* domain, const std::vector<Field>& schema, const einfold_options& o,
                             Budget& budget);
FoldOutput chain_fold(Context& ctx, const FoldD& f, const std::vector<const Relation*>& operands,
                      const std::vector<Field>& schema, const einfold_options& o, Budget& budget);
FoldOutput fused_pipeline(Context& ctx, const PipelineD& p, const Relation& q, const Relation& k, const Relation& v,
                          const std::vector<Field>& schema, const einfold_options& o, Budget& budget);

// The gradients of an attention-shaped pipeline's result (product scores,
// weights exp(s - MAX(s)), normalised over the kept groups) with respect to
// the factors of q, k and v, given d_out keyed as the result: per operand a
// row per placed cell, its key columns and the gradient.
struct GradientOutput {
  std::vector<OutBatch> batches[3];
  std::vector<Field> schemas[3];
};
GradientOutput pipeline_backward(Context& ctx, const PipelineD& p, const Relation& q, const Relation& k,
                                 const Relation& v, const Relation& d_out, const einfold_options& o);

}  // namespace ef
