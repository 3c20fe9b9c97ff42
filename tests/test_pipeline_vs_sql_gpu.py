"""The reference's property test of the fused pipeline against SQL
(crates/einfold-kernels/tests/pipeline_vs_sql.rs), on the B200 path.

Cases are drawn as that test draws them (pipeline_vs_sql.rs:138-497), seed by
seed from its default seed, with the SplitMix64 stream of einfold's test
kit: tables q([b,] t, d, x), k([b,] t, d, x) and v([b,] t, [c,] x) with
random extents; scores SUM(q.x * k.x) over d, or the sum of a row expression
of q.x and k.x (a Gaussian kernel's -power(q.x - k.x, 2) among them), or,
without d, over a CROSS JOIN's one row a pair; scaled by a constant or not;
under none, one or two conditions between q.t and k.t; weights
exp(s - MAX(s) OVER (PARTITION BY [b,] i)), exp(s), 1/(1 + exp(-s)),
1/(1 + s^2), or s itself for a sum nothing normalizes; normalized by the
kept groups' weights, by the joined rows', or not at all. Values spread
widely; some are NaN, +-inf or +-1e300, some rows' scores are all -inf or
-inf beside a NaN; some tables miss, repeat or NULL a row. Every draw is
made in the reference's order.

The SQL is evaluated here, independently of the kernels and of oracle/.
The invariants (pipeline_vs_sql.rs:25-40), in both product forms:

1. it runs when every table is complete, the producer reads both operands
   and no value is special; otherwise it may decline;
2. the same rows as SQL;
3. NaN where SQL gives NaN, the same infinity, otherwise within
   1e-9 max|v.x| (an average), or 1e-9 sum|w v.x| of the group (a sum);
4. other batchings give the same bits.
"""
import math

import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle

pytestmark = pytest.mark.gpu

SEED, CASES = 0xA77E0001, 150
FORMS = (K.Precision.FP64, K.Precision.SPLIT)
EQ = ir.Dimension(ir.KeyEquality.EQUAL)
COMPARISONS = [ir.Comparison.LESS, ir.Comparison.LESS_OR_EQUAL, ir.Comparison.GREATER,
               ir.Comparison.GREATER_OR_EQUAL]


class Draws(oracle.Rng):
    """einfold_testkit::Rng, its words drawn in bulk by the oracle's C fill
    of the same stream and handed out one at a time."""

    def __init__(self, seed, salt):
        super().__init__(seed, salt)
        self._buf, self._i = [], 0

    def next_u64(self):
        if self._i == len(self._buf):
            self._buf, self._i = oracle.Rng.u64s(self, 1 << 15).tolist(), 0
        v = self._buf[self._i]
        self._i += 1
        return v


class Table:
    """Rows of (int64 keys, a nullable DOUBLE x)."""

    def __init__(self, names, extents):
        self.names = list(names)
        self.rows = []
        cells = int(np.prod(extents)) if extents else 1
        for c in range(cells):
            keys = [0] * len(extents)
            for s in range(len(extents) - 1, -1, -1):
                keys[s] = c % extents[s]
                c //= extents[s]
            self.rows.append([keys, 0.0])

    def schema(self):
        return pa.schema([pa.field(n, pa.int64(), nullable=False) for n in self.names] + [pa.field("x", pa.float64())])

    def partitions(self, rng):
        """The rows shuffled, in partitions of batches of random sizes,
        concatenated in partition order (pipeline_vs_sql.rs:90-119)."""
        order = list(range(len(self.rows)))
        for i in range(len(order) - 1, 0, -1):
            j = rng.below(i + 1)
            order[i], order[j] = order[j], order[i]
        parts = [[] for _ in range(1 + rng.below(3))]
        start = 0
        schema = self.schema()
        while start < len(order):
            end = min(start + 1 + rng.below(300), len(order))
            rows = [self.rows[r] for r in order[start:end]]
            cols = [pa.array([r[0][c] for r in rows], type=pa.int64()) for c in range(len(self.names))]
            cols.append(pa.array([r[1] for r in rows], type=pa.float64()))
            parts[rng.below(len(parts))].append(pa.RecordBatch.from_arrays(cols, schema=schema))
            start = end
        flat = [b for p in parts for b in p]
        return flat or [pa.RecordBatch.from_arrays([pa.array([], type=f.type) for f in schema], schema=schema)]


def value(rng, spread, specials):
    if specials and rng.chance(0.004):
        return [math.nan, math.inf, -math.inf, 1e300, -1e300][rng.below(5)]
    return (2.0 * rng.unit() - 1.0) * spread


# A row value: (IR, SQL evaluation over q.x and k.x, reads both operands).
def _pow2(a):
    return a * a


ROW_VALUES = {
    "product": (None, lambda q, k: q * k),
    "gauss": (lambda Q, Kc, lit: Q.binary(ir.Binary.SUBTRACT, Kc).binary(ir.Binary.POWER, lit(2.0)).unary(
        ir.Unary.NEGATE), lambda q, k: -_pow2(q - k)),
    "laplace": (lambda Q, Kc, lit: Q.binary(ir.Binary.SUBTRACT, Kc).unary(ir.Unary.ABS).unary(ir.Unary.NEGATE),
                lambda q, k: -abs(q - k)),
    "times": (lambda Q, Kc, lit: Q.binary(ir.Binary.MULTIPLY, Kc), lambda q, k: q * k),
    "mixed": (lambda Q, Kc, lit: Q.binary(ir.Binary.MULTIPLY, Kc.binary(ir.Binary.DIVIDE, lit(4.0)).unary(
        ir.Unary.EXP)).binary(ir.Binary.ADD, lit(0.5)), lambda q, k: q * _exp(k / 4.0) + 0.5),
    "exp_q": (lambda Q, Kc, lit: Q.unary(ir.Unary.EXP), lambda q, k: _exp(q)),
    "abs_k": (lambda Q, Kc, lit: Kc.unary(ir.Unary.ABS).unary(ir.Unary.NEGATE), lambda q, k: -abs(k)),
    "half": (lambda Q, Kc, lit: lit(0.5), lambda q, k: 0.5),
}


def _exp(x):
    if x != x:
        return x
    try:
        return math.exp(x)
    except OverflowError:
        return math.inf


def row_value(rng):
    if rng.chance(0.1):
        return ["exp_q", "abs_k", "half"][min(rng.below(3), 2)]
    return {0: "product", 1: "product", 2: "gauss", 3: "laplace", 4: "times"}.get(rng.below(6), "mixed")


# ---- cases (pipeline_vs_sql.rs:193-497) --------------------------------------

class Case:
    pass


def draw_case(rng):
    c = Case()
    c.cross = rng.chance(0.25)
    c.nq = 1 + rng.below(150)
    c.nk = 1 + rng.below(150)
    c.nd = 1 if c.cross else 1 + rng.below(6)
    c.channels = 1 + rng.below(4) if rng.chance(0.6) else None
    c.batch = 1 + rng.below(3) if rng.chance(0.4) else None
    specials = rng.chance(0.3)
    spread = [1.0, 4.0, 12.0][rng.below(3)]
    keys = ["t"] if c.cross else ["t", "d"]
    eq, ek = ([c.nq], [c.nk]) if c.cross else ([c.nq, c.nd], [c.nk, c.nd])
    b0 = 1 if c.batch else 0
    if c.batch:
        keys = ["b"] + keys
        eq, ek = [c.batch] + eq, [c.batch] + ek
    c.q, c.k = Table(keys, eq), Table(keys, ek)
    for r in c.q.rows + c.k.rows:
        r[1] = value(rng, spread, specials)
    vn, ve = (["t", "c"], [c.nk, c.channels]) if c.channels else (["t"], [c.nk])
    if c.batch:
        vn, ve = ["b"] + vn, [c.batch] + ve
    c.v = Table(vn, ve)
    for r in c.v.rows:
        r[1] = value(rng, 1.0, specials)
    # Rows of q whose scores are -inf: all, or those with the first 64 keys
    # beside a NaN score (row t·nd + d is (t, d) of the first batch).
    at = lambda t, d: t * c.nd + d  # noqa: E731
    target = rng.below(c.nq)
    extremes = rng.below(6)
    if extremes == 0:
        c.q.rows[at(target, 0)][1] = -math.inf
        for j in range(c.nk):
            x = c.k.rows[at(j, 0)]
            x[1] = None if x[1] is None else abs(x[1]) + 0.1
    elif extremes == 1 and c.nk > 64:
        c.q.rows[at(target, 0)][1] = -1e300
        for j in range(64):
            c.k.rows[at(j, 0)][1] = 1e300
        c.k.rows[at(rng.below(64), c.nd - 1)][1] = math.nan
    complete = not rng.chance(0.15)
    if not complete:
        t = [c.q, c.k, c.v][rng.below(3)]
        r = rng.below(len(t.rows))
        kind = rng.below(3)
        if kind == 0:
            del t.rows[r]
        elif kind == 1:
            t.rows.append([list(t.rows[r][0]), t.rows[r][1]])
        else:
            t.rows[r][1] = None
    finite = [abs(r[1]) for r in c.v.rows if r[1] is not None and math.isfinite(r[1])]
    c.v_scale = max(finite, default=0.0)

    di, dj = (0, 1) if c.cross else (0, 2)
    producer_dims = (2 if c.cross else 3) + b0
    db, dc = producer_dims - 1, producer_dims
    x = len(keys)
    if c.cross:
        while True:
            c.row = row_value(rng)
            if c.row != "product":
                break
    else:
        c.row = row_value(rng)
    reads_both = c.row not in ("exp_q", "abs_k", "half")

    def operand(own):
        ks = [(d, i + b0) for i, d in enumerate(own)]
        if c.batch:
            ks = [(db, 0)] + ks
        return ir.Operand(ks, len(own) + b0)

    ops = [operand([di]), operand([dj])] if c.cross else [operand([di, 1]), operand([dj, 1])]
    outs = [ir.Output(di), ir.Output(dj)]
    if c.batch:
        outs = [ir.Output(db)] + outs
    build, c.row_sql = ROW_VALUES[c.row]
    Q, Kc, lit = ir.Expression.column(0, x), ir.Expression.column(1, x), ir.Expression.literal
    row = ir.RowValue.PRODUCT if build is None else ir.RowValue(build(Q, Kc, lit))
    producer = ir.Fold([EQ] * producer_dims, ops, outs, row)
    c.conditions = []
    conds = []
    for _ in range([0, 1, 1, 2][rng.below(4)]):
        cmp = COMPARISONS[rng.below(4)]
        offset = 0 if rng.chance(0.3) else rng.below(81) - 40
        q_left = rng.chance(0.5)
        left, right = (di, dj) if q_left else (dj, di)
        conds.append(ir.Condition(left, cmp, right, offset))
        c.conditions.append((q_left, cmp, offset))
    producer = producer.with_conditions(conds)
    scale_kind = rng.below(3)
    scale = [ir.Scale.one(), ir.Scale.times(-0.7), ir.Scale.over(8.0)][scale_kind]
    c.scale = [lambda s: s, lambda s: s * -0.7, lambda s: s / 8.0][scale_kind]
    c.normalizer = [ir.Normalizer.KEPT_GROUPS, ir.Normalizer.JOINED_ROWS, ir.Normalizer.NONE][rng.below(3)]

    def p():
        e = ir.Expression.column(0, 0)
        if scale_kind == 1:
            return e.binary(ir.Binary.MULTIPLY, lit(-0.7))
        if scale_kind == 2:
            return e.binary(ir.Binary.DIVIDE, lit(8.0))
        return e

    def one_over(e):
        return lit(1.0).binary(ir.Binary.DIVIDE, lit(1.0).binary(ir.Binary.ADD, e))

    w = rng.below(5)
    if w == 0:
        weight, c.weight = ir.Weight.of_expression(one_over(p().unary(ir.Unary.NEGATE).unary(ir.Unary.EXP))), "logistic"
    elif w == 1:
        weight, c.weight = ir.Weight.of_expression(one_over(p().binary(ir.Binary.MULTIPLY, p()))), "cauchy"
    elif w == 2 and c.normalizer == ir.Normalizer.NONE:
        weight, c.weight = ir.Weight.of_expression(p()), "score"
    elif w in (2, 3):
        weight, c.weight = ir.Weight.exp(scale, ir.Shift.KEPT_MAXIMUM), "softmax"
    else:
        weight, c.weight = ir.Weight.exp(scale, ir.Shift.NONE), "exp"
    if c.channels:
        values, outputs = operand([dj, dc]), [di, dc]
    else:
        values, outputs = operand([dj]), [di]
    if c.batch:
        outputs = [db] + outputs
    c.pipeline = ir.Pipeline(producer, weight, [EQ] if c.channels else [], values, outputs, c.normalizer)
    c.complete = complete and reads_both and not specials and extremes > 1
    return c


# ---- SQL's answer, evaluated here --------------------------------------------

def div(a, b):
    """IEEE division, as SQL's DOUBLE division."""
    if b == 0.0:
        if a == 0.0 or a != a:
            return math.nan
        return math.copysign(math.inf, a) * math.copysign(1.0, b)
    return a / b


def sql_max(xs):
    """MAX over DOUBLEs: NULLs ignored, NaN the largest."""
    xs = [x for x in xs if x is not None]
    if not xs:
        return None
    if any(x != x for x in xs):
        return math.nan
    return max(xs)


def sql_sum(xs):
    xs = [x for x in xs if x is not None]
    if not xs:
        return None
    s = 0.0
    for x in xs:
        s += x
    return s


def holds(cmp, a, b):
    return {ir.Comparison.LESS: a < b, ir.Comparison.LESS_OR_EQUAL: a <= b, ir.Comparison.GREATER: a > b,
            ir.Comparison.GREATER_OR_EQUAL: a >= b}[cmp]


def sql(c):
    """The pipeline's rows: {(b?, i, c?): (value or None, scale of its rounding)}."""
    row = c.row_sql
    reads = {"exp_q": (True, False), "abs_k": (False, True), "half": (False, False)}.get(c.row, (True, True))
    bq = 1 if c.batch else 0

    def allowed(qt, kt):
        for q_left, cmp, off in c.conditions:
            if not (holds(cmp, qt, kt + off) if q_left else holds(cmp, kt, qt + off)):
                return False
        return True

    def rv(qx, kx):
        if (reads[0] and qx is None) or (reads[1] and kx is None):
            return None
        return row(qx if qx is not None else 0.0, kx if kx is not None else 0.0)

    # Scores: per (b, i, j) the SUM over d (one list a pair of rows under a
    # CROSS JOIN, where a repeated row repeats the pair).
    by_k = {}
    for kr in c.k.rows:
        key = (kr[0][0] if c.batch else 0, kr[0][bq + 1] if not c.cross else 0)
        by_k.setdefault(key, []).append(kr)
    scores = []  # (b, i, j, s)
    if c.cross:
        for qr in c.q.rows:
            b = qr[0][0] if c.batch else 0
            for kr in by_k.get((b, 0), ()):
                if allowed(qr[0][bq], kr[0][bq]):
                    v = rv(qr[1], kr[1])
                    scores.append((b, qr[0][bq], kr[0][bq], None if v is None else c.scale(v)))
    else:
        groups = {}
        for qr in c.q.rows:
            b = qr[0][0] if c.batch else 0
            for kr in by_k.get((b, qr[0][bq + 1]), ()):
                if allowed(qr[0][bq], kr[0][bq]):
                    groups.setdefault((b, qr[0][bq], kr[0][bq]), []).append(rv(qr[1], kr[1]))
        for (b, i, j), terms in groups.items():
            s = sql_sum(terms)
            scores.append((b, i, j, None if s is None else c.scale(s)))
    # Weights.
    if c.weight == "softmax":
        part = {}
        for b, i, j, s in scores:
            part.setdefault((b, i), []).append(s)
        mx = {k: sql_max(v) for k, v in part.items()}
    weights = []
    for b, i, j, s in scores:
        if s is None:
            w = None
        elif c.weight == "logistic":
            w = div(1.0, 1.0 + _exp(-s))
        elif c.weight == "cauchy":
            w = div(1.0, 1.0 + s * s)
        elif c.weight == "score":
            w = s
        elif c.weight == "softmax":
            m = mx[(b, i)]
            w = None if m is None else _exp(s - m)
        else:
            w = _exp(s)
        weights.append((b, i, j, w))
    # weights JOIN v ON j = v.t [AND b = v.b], grouped by (b, i, c).
    by_v = {}
    for vr in c.v.rows:
        b = vr[0][0] if c.batch else 0
        by_v.setdefault((b, vr[0][bq]), []).append(vr)
    joined = {}
    z = {}
    for b, i, j, w in weights:
        z.setdefault((b, i), []).append(w)
        for vr in by_v.get((b, j), ()):
            ch = vr[0][bq + 1] if c.channels else None
            joined.setdefault((b, i, ch), []).append((w, vr[1]))
    out = {}
    for (b, i, ch), pairs in joined.items():
        prods = [None if (w is None or x is None) else w * x for w, x in pairs]
        num = sql_sum(prods)
        if c.normalizer == ir.Normalizer.KEPT_GROUPS:
            den = sql_sum(z[(b, i)])
            val = None if (num is None or den is None) else div(num, den)
            scale = c.v_scale
        elif c.normalizer == ir.Normalizer.JOINED_ROWS:
            den = sql_sum([w for w, _ in pairs])
            val = None if (num is None or den is None) else div(num, den)
            scale = c.v_scale
        else:
            val = num
            mags = sql_sum([None if p is None else abs(p) for p in prods])
            scale = mags if mags is not None else 0.0
        key = ((b,) if c.batch else ()) + (i,) + ((ch,) if c.channels else ())
        out[key] = (val, scale)
    return out


# ---- the kernel's answers and the invariants (pipeline_vs_sql.rs:531-623) ----

HOST = K.Host(K.FloatKeys.SIGNED_ZEROS_EQUAL)


def run(c, rng):
    """The pipeline in each product form over one random batching of the
    tables, or None where it declined."""
    rels = [K.Relation(t.schema(), t.partitions(rng)) for t in (c.q, c.k, c.v)]
    rng.below(12)  # threads: one device here
    out = {}
    for f in FORMS:
        got = K.pipeline(c.pipeline, rels, options=K.Options(host=HOST, precision=f))
        out[f] = None if got is None else got.batches
    return out


def rows_of(batches):
    out = {}
    for b in batches:
        n = b.num_columns - 1
        keys = [b.column(i).to_pylist() for i in range(n)]
        vals = b.column(n).to_pylist()
        for r in range(b.num_rows):
            out[tuple(k[r] for k in keys)] = vals[r]
    return out


def bits(rows):
    return sorted((k, None if v is None else np.float64(v).view(np.uint64).item()) for k, v in rows.items())


def same(ours, theirs, bound):
    if ours is None or theirs is None:
        return ours is None and theirs is None
    if ours != ours or theirs != theirs:
        return ours != ours and theirs != theirs
    if math.isinf(ours) or math.isinf(theirs):
        return ours == theirs
    return abs(ours - theirs) <= bound


def test_pipelines_match_sql():
    stats = dict(cases=0, ran=0, declined=0)
    failures = []
    for i in range(CASES):
        seed = SEED + i
        rng = Draws(seed, 0)
        c = draw_case(rng)
        stats["cases"] += 1
        try:
            ours = run(c, rng)
            if c.complete:
                assert all(ours[f] is not None for f in FORMS), "declined complete inputs"
            if all(ours[f] is None for f in FORMS):
                stats["declined"] += 1
                continue
            stats["ran"] += 1
            again = run(c, rng)
            theirs = sql(c)
            for f in FORMS:
                if ours[f] is None:
                    continue
                assert again[f] is not None, f"ran on one batching and declined on another ({f.name})"
                got = rows_of(ours[f])
                assert bits(got) == bits(rows_of(again[f])), f"two arrival orders gave different bits ({f.name})"
                assert sorted(got) == sorted(theirs), f"{len(got)} rows, SQL has {len(theirs)} ({f.name})"
                for key, v in got.items():
                    want, scale = theirs[key]
                    assert same(v, want, 1e-9 * scale), f"row {key} = {v}, SQL has {want} ({f.name})"
        except AssertionError as e:
            failures.append(f"seed {seed}: {e}")
    print(stats)
    assert not failures, "\n".join(failures[:20])
