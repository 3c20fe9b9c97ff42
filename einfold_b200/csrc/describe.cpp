// Parsing of fold and pipeline descriptions, and result schemas.
#include <cstring>

#include "fold.h"

namespace ef {

static std::vector<ExprNode> parse_expression(const einfold_expression& e) {
  std::vector<ExprNode> out;
  int depth = 0;
  for (int32_t i = 0; i < e.n_nodes; i++) {
    const einfold_expr_node& n = e.nodes[i];
    ExprNode x{n.kind, n.a, n.b, n.value};
    if (n.kind == 0 || n.kind == 1) depth++;
    else if (n.kind == 2) {
      if (depth < 1 || n.a < 0 || n.a > 3) fail(EINFOLD_INVALID, "a malformed expression");
    } else if (n.kind == 3) {
      if (depth < 2 || n.a < 0 || n.a > 4) fail(EINFOLD_INVALID, "a malformed expression");
      depth--;
    } else {
      fail(EINFOLD_INVALID, "an expression node of kind %d", n.kind);
    }
    if (depth > 60) fail(EINFOLD_INVALID, "an expression deeper than 60");
    out.push_back(x);
  }
  if (!out.empty() && depth != 1) fail(EINFOLD_INVALID, "a malformed expression");
  return out;
}

static OperandD parse_operand(const einfold_operand& o) {
  OperandD op;
  for (int32_t i = 0; i < o.n_keys; i++) op.keys.push_back({o.keys[i].dimension, o.keys[i].column});
  op.factor = o.factor;
  return op;
}

FoldD parse_fold(const einfold_fold_desc* d) {
  if (!d) fail(EINFOLD_INVALID, "no fold");
  FoldD f;
  int n = d->n_dimensions;
  for (int i = 0; i < n; i++) f.equality.push_back(d->equality ? d->equality[i] : 0);
  for (int i = 0; i < d->n_operands; i++) f.operands.push_back(parse_operand(d->operands[i]));
  for (int i = 0; i < d->n_outputs; i++)
    f.outputs.push_back({d->outputs[i].dimension, d->outputs[i].domain_column, d->outputs[i].domain_equality});
  f.row_expr = d->row_is_expression != 0;
  if (f.row_expr) f.row = parse_expression(d->row);
  if (d->domain) {
    DomainD dom;
    for (int i = 0; i < d->domain->n_carry; i++) dom.carry.push_back(d->domain->carry[i]);
    dom.has_missing = d->domain->has_missing != 0;
    dom.missing = d->domain->missing;
    f.domain = dom;
  }
  for (int i = 0; i < d->n_conditions; i++) {
    const einfold_condition& c = d->conditions[i];
    if (c.comparison < 0 || c.comparison > 3) fail(EINFOLD_INVALID, "a comparison of kind %d", c.comparison);
    f.conditions.push_back({c.left, c.comparison, c.right, c.offset});
  }
  // Fold::try_new's rules.
  for (size_t i = 0; i < f.operands.size(); i++) {
    std::vector<bool> seen(n, false);
    for (auto& k : f.operands[i].keys) {
      if (k.dim < 0 || k.dim >= n) fail(EINFOLD_INVALID, "operand %zu names dimension %d, of %d", i, k.dim, n);
      if (seen[k.dim]) fail(EINFOLD_INVALID, "operand %zu holds dimension %d twice", i, k.dim);
      seen[k.dim] = true;
    }
  }
  for (int dd = 0; dd < n; dd++) {
    bool any = false;
    for (auto& op : f.operands) any |= op.holds(dd);
    if (!any) fail(EINFOLD_INVALID, "no operand holds dimension %d", dd);
  }
  if (!f.row_expr) {
    bool any = false;
    for (auto& op : f.operands) any |= op.factor >= 0;
    if (!any) fail(EINFOLD_INVALID, "no operand has a factor");
  } else {
    for (auto& oc : f.row_columns())
      if (oc.first < 0 || oc.first >= (int)f.operands.size())
        fail(EINFOLD_INVALID, "the row expression reads operand %d, of %zu", oc.first, f.operands.size());
  }
  std::vector<bool> seen(n, false);
  for (auto& o : f.outputs) {
    if (o.dim < 0 || o.dim >= n) fail(EINFOLD_INVALID, "output dimension %d, of %d", o.dim, n);
    if (seen[o.dim]) fail(EINFOLD_INVALID, "dimension %d is output twice", o.dim);
    seen[o.dim] = true;
    if ((o.domain_col >= 0) != f.domain.has_value())
      fail(EINFOLD_INVALID, "output of dimension %d has a domain key exactly when the fold has a domain", o.dim);
  }
  for (auto& c : f.conditions) {
    if (c.left < 0 || c.right < 0 || c.left >= n || c.right >= n)
      fail(EINFOLD_INVALID, "a condition compares dimensions %d and %d, of %d", c.left, c.right, n);
    if (c.left == c.right) fail(EINFOLD_INVALID, "a condition compares dimension %d with itself", c.left);
  }
  return f;
}

PipelineD parse_pipeline(const einfold_pipeline_desc* d) {
  if (!d) fail(EINFOLD_INVALID, "no pipeline");
  PipelineD p;
  p.producer = parse_fold(d->producer);
  p.weight_expr = d->weight_is_expression != 0;
  p.scale_kind = d->scale_kind;
  p.scale_c = d->scale_c;
  p.shift = d->shift;
  p.normalizer = d->normalizer;
  if (p.weight_expr) p.weight = parse_expression(d->weight);
  for (int i = 0; i < d->n_dimensions; i++) p.equality.push_back(d->equality ? d->equality[i] : 0);
  p.values = parse_operand(d->values);
  for (int i = 0; i < d->n_outputs; i++) p.outputs.push_back(d->outputs[i]);
  // Pipeline::try_new's rules.
  const FoldD& pr = p.producer;
  if (pr.domain) fail(EINFOLD_INVALID, "a pipeline's producer is a SUM of products or of a row expression, with no domain");
  if (p.weight_expr)
    for (auto& n : p.weight)
      if (n.kind == 0 && !(n.a == 0 && n.b == 0))
        fail(EINFOLD_INVALID, "a pipeline's weight reads only the producer's value");
  if (p.values.factor < 0) fail(EINFOLD_INVALID, "a pipeline's values operand has no factor");
  int own = pr.n_dims(), n = own + (int)p.equality.size();
  std::vector<bool> held(n, false), output(n, false);
  for (auto& k : p.values.keys) {
    if (k.dim < 0 || k.dim >= n || (k.dim < own && pr.output_of(k.dim) < 0))
      fail(EINFOLD_INVALID, "the values operand holds dimension %d, not an output", k.dim);
    if (held[k.dim]) fail(EINFOLD_INVALID, "the values operand holds dimension %d twice", k.dim);
    held[k.dim] = true;
  }
  for (int dd : p.outputs) {
    if (dd < 0 || dd >= n || (dd < own && pr.output_of(dd) < 0))
      fail(EINFOLD_INVALID, "output dimension %d is not a producer output", dd);
    if (output[dd]) fail(EINFOLD_INVALID, "dimension %d is output twice", dd);
    output[dd] = true;
  }
  for (auto& o : pr.outputs)
    if (!output[o.dim] && !held[o.dim]) fail(EINFOLD_INVALID, "producer output %d is summed but not joined", o.dim);
  for (int dd = own; dd < n; dd++)
    if (!held[dd]) fail(EINFOLD_INVALID, "the values operand doesn't hold dimension %d", dd);
  return p;
}

static const Field& field_at(const std::vector<Field>& s, int col, const char* what) {
  if (col < 0 || col >= (int)s.size()) fail(EINFOLD_INVALID, "column %d of %s with %zu", col, what, s.size());
  return s[col];
}

static bool same_type(const Field& a, const Field& b) {
  if (a.format != b.format) return false;
  if (!!a.dictionary != !!b.dictionary) return false;
  if (a.dictionary) return same_type(*a.dictionary, *b.dictionary);
  return true;
}

static Field named(const Field& f, size_t i) {
  Field g = f;
  g.name = std::to_string(i);
  return g;
}

std::vector<Field> fold_schema(const FoldD& f, const std::vector<const std::vector<Field>*>& operands,
                               const std::vector<Field>* domain) {
  bool chain = f.operands.size() == 3 && !f.domain;
  if (!(f.operands.size() == 2 || chain) || operands.size() != f.operands.size())
    fail(EINFOLD_INVALID, "EinFold computes folds of two operands, or chains of three, not %zu", f.operands.size());
  if (f.domain.has_value() != (domain != nullptr))
    fail(EINFOLD_INVALID, "a domain relation must be given exactly when the fold has a domain");
  std::vector<std::pair<int, int>> values;
  if (!f.row_expr) {
    for (size_t o = 0; o < f.operands.size(); o++) {
      if (f.operands[o].factor < 0) fail(EINFOLD_INVALID, "EinFold doesn't compute masks yet");
      values.push_back({(int)o, f.operands[o].factor});
    }
  } else {
    values = f.row_columns();
  }
  for (auto& v : values) {
    const Field& fv = field_at(*operands[v.first], v.second, "an input");
    if (fv.format != "g" || fv.dictionary) fail(EINFOLD_INVALID, "EinFold's values must be Float64, not %s", fv.format.c_str());
  }
  std::vector<const Field*> types(f.n_dims(), nullptr);
  for (size_t o = 0; o < f.operands.size(); o++)
    for (auto& k : f.operands[o].keys) {
      const Field& kf = field_at(*operands[o], k.col, "an input");
      if (!types[k.dim]) types[k.dim] = &kf;
      else if (!same_type(*types[k.dim], kf))
        fail(EINFOLD_INVALID, "dimension %d's columns have types %s and %s", k.dim, types[k.dim]->format.c_str(),
             kf.format.c_str());
    }
  std::vector<Field> fields;
  if (f.domain) {
    for (auto& o : f.outputs) {
      const Field& kf = field_at(*domain, o.domain_col, "the domain");
      if (!same_type(kf, *types[o.dim]))
        fail(EINFOLD_INVALID, "the domain's column for dimension %d is %s, the operands' %s", o.dim, kf.format.c_str(),
             types[o.dim]->format.c_str());
    }
    for (int c : f.domain->carry) fields.push_back(named(field_at(*domain, c, "the domain"), fields.size()));
  } else {
    for (auto& o : f.outputs) fields.push_back(named(*types[o.dim], fields.size()));
  }
  Field v;
  v.format = "g";
  v.kind = Kind::Float64;
  v.nullable = !f.domain || !f.domain->has_missing;
  v.name = std::to_string(fields.size());
  fields.push_back(v);
  return fields;
}

std::vector<Field> pipeline_schema(const PipelineD& p, const std::vector<const std::vector<Field>*>& inputs) {
  std::vector<const std::vector<Field>*> two = {inputs[0], inputs[1]};
  std::vector<Field> producer = fold_schema(p.producer, two, nullptr);
  const std::vector<Field>& vs = *inputs[2];
  const Field& factor = field_at(vs, p.values.factor, "the values operand");
  if (factor.format != "g") fail(EINFOLD_INVALID, "EinFold factors must be Float64, not %s", factor.format.c_str());
  auto key = [&](int d) -> const Field& {
    int o = p.producer.output_of(d);
    if (o >= 0) return producer[o];
    return field_at(vs, p.values.column_of(d), "the values operand");
  };
  for (auto& k : p.values.keys) {
    const Field& want = key(k.dim);
    const Field& got = field_at(vs, k.col, "the values operand");
    if (!same_type(want, got))
      fail(EINFOLD_INVALID, "dimension %d's columns have types %s and %s", k.dim, want.format.c_str(), got.format.c_str());
  }
  std::vector<Field> fields;
  for (int d : p.outputs) fields.push_back(named(key(d), fields.size()));
  Field v;
  v.format = "g";
  v.kind = Kind::Float64;
  v.nullable = true;
  v.name = std::to_string(fields.size());
  fields.push_back(v);
  return fields;
}

}  // namespace ef
