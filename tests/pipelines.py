"""Attention-shaped pipelines and their tables for the parity tests, after
the cases of crates/einfold-kernels/tests/pipeline_vs_sql.rs: q([b,] t, d, x),
k([b,] t, d, x), v([b,] t, [c,] x), scores SUM(q.x * k.x) over d (or a row
expression of q.x and k.x), conditions between q.t and k.t, weights a
softmax or an expression of the score, and a normalizer."""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import pyarrow as pa

from einfold_b200 import ir
from oracle import oracle
from tests.tables import complete

E = ir.Dimension(ir.KeyEquality.EQUAL)
I, D, J, B = 0, 1, 2, 3  # dimensions: q.t, d, k.t, the batch key


@dataclass
class Case:
    pipeline: ir.Pipeline
    q: Tuple[pa.Schema, List[pa.RecordBatch]]
    k: Tuple[pa.Schema, List[pa.RecordBatch]]
    v: Tuple[pa.Schema, List[pa.RecordBatch]]
    v_scale: float


def gaussian_scores() -> ir.Expression:
    """-power(q.x - k.x, 2): a Gaussian kernel's exponent, summed over d."""
    diff = ir.Expression.column(0, -1).binary(ir.Binary.SUBTRACT, ir.Expression.column(1, -1))
    return diff.binary(ir.Binary.POWER, ir.Expression.literal(2.0)).unary(ir.Unary.NEGATE)


def sigmoid_weight() -> ir.Expression:
    """1 / (1 + exp(-s))."""
    s = ir.Expression.column(0, 0)
    one = ir.Expression.literal(1.0)
    return one.binary(ir.Binary.DIVIDE, one.binary(ir.Binary.ADD, s.unary(ir.Unary.NEGATE).unary(ir.Unary.EXP)))


def cauchy_weight() -> ir.Expression:
    """1 / (1 + s * s)."""
    s = ir.Expression.column(0, 0)
    one = ir.Expression.literal(1.0)
    return one.binary(ir.Binary.DIVIDE, one.binary(ir.Binary.ADD, s.binary(ir.Binary.MULTIPLY, s)))


def _fix_columns(e: ir.Expression, factor: int) -> ir.Expression:
    """Column -1 of an operand means its factor column."""
    if e.kind == "column":
        return ir.Expression.column(e.operand, factor if e.col == -1 else e.col)
    if e.kind == "literal":
        return e
    args = [_fix_columns(a, factor) for a in e.args]
    return ir.Expression(e.kind, op=e.op, args=args)


def attention(l: int, d: int = 8, nb: Optional[int] = None, c: Optional[int] = None, lk: Optional[int] = None,
              conditions: Sequence[Tuple[ir.Comparison, int]] = (), mirrored: bool = False,
              weight: Optional[ir.Weight] = None, normalizer: ir.Normalizer = ir.Normalizer.KEPT_GROUPS,
              scores: Optional[ir.Expression] = None,
              q_value: Optional[Callable[[int], np.ndarray]] = None,
              k_value: Optional[Callable[[int], np.ndarray]] = None,
              v_value: Optional[Callable[[int], np.ndarray]] = None,
              seed: int = 7, batches: int = 3) -> Case:
    """A pipeline over l query and lk (= l) key positions, d features, nb
    batches (a batch key b, first in every table) and c value columns (a
    pipeline dimension c) or one."""
    rng = oracle.Rng.seeded(seed, 0)
    lk = l if lk is None else lk
    b0 = 1 if nb else 0
    pre_n, pre_e = (["b"], [nb]) if nb else ([], [])
    qv = q_value or (lambda n: rng.units(n))
    kv = k_value or (lambda n: np.full(n, 0.5))
    vv = v_value or (lambda n: np.ones(n))
    nq = (nb or 1) * l * d
    nk = (nb or 1) * lk * d
    q = complete(pre_n + ["t", "d"], pre_e + [l, d], qv(nq), rng, batches=batches)
    k = complete(pre_n + ["t", "d"], pre_e + [lk, d], kv(nk), rng, batches=batches)
    v_names = pre_n + ["t"] + (["c"] if c else [])
    v_ext = pre_e + [lk] + ([c] if c else [])
    v = complete(v_names, v_ext, vv(int(np.prod(v_ext))), rng, batches=batches)

    def operand(own):
        keys = [ir.Key(dd, i + b0) for i, dd in enumerate(own)]
        if nb:
            keys.insert(0, ir.Key(B, 0))
        return ir.Operand(keys, len(own) + b0)

    dims = [E, E, E] + ([E] if nb else [])
    outputs = [ir.Output(I), ir.Output(J)]
    kept = [I]
    if nb:
        outputs.insert(0, ir.Output(B))
        kept.insert(0, B)
    row = ir.RowValue.PRODUCT if scores is None else ir.RowValue(_fix_columns(scores, 2 + b0))
    producer = ir.Fold(dims, [operand([I, D]), operand([J, D])], outputs, row)
    conds = [ir.Condition(J, ir.Comparison(cmp).mirrored(), I, -off) if mirrored else ir.Condition(I, cmp, J, off)
             for cmp, off in conditions]
    if conds:
        producer = producer.with_conditions(conds)
    own = len(dims)
    vkeys = [ir.Key(J, b0)] + ([ir.Key(own, b0 + 1)] if c else [])
    if nb:
        vkeys.insert(0, ir.Key(B, 0))
    values = ir.Operand(vkeys, len(v_names))
    outs = kept + ([own] if c else [])
    p = ir.Pipeline(producer, weight or ir.Weight.exp(), [E] if c else [], values, outs, normalizer)
    vals = np.concatenate([b.column(b.num_columns - 1).to_numpy(zero_copy_only=False) for b in v[1]]) if v[1] else [0]
    fin = np.asarray(vals, np.float64)
    fin = fin[np.isfinite(fin)]
    return Case(p, q, k, v, float(np.max(np.abs(fin))) if len(fin) else 0.0)


def run_oracle(case: Case, threads: int = 4):
    out_schema = oracle.pipeline_schema(case.pipeline, [case.q[0], case.k[0], case.v[0]])
    return oracle.pipeline(case.pipeline, case.q[1], case.k[1], case.v[1], out_schema, oracle.Options(threads=threads))
