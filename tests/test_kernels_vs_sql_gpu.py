"""The reference's property test of the kernels against SQL
(crates/einfold-kernels/tests/kernels_vs_sql.rs), on the B200 path.

Cases are drawn as that test draws them (kernels_vs_sql.rs:163-558), seed by
seed from its default seed, with the SplitMix64 stream of einfold's test kit:
folds of two operands over one to four dimensions, keys BIGINT (from -1),
non-negative BIGINT, UInt64 (with 2^63, beyond BIGINT), VARCHAR, DOUBLE
(0.0, -0.0, NaN, 2.5, -1.0) or dictionary-encoded VARCHAR (NULL as a NULL
dictionary value), compared with = or IS NOT DISTINCT FROM; random outputs;
half the time a domain (each key matched by either equality, a random
default or none). Tables have NULL keys, duplicate key tuples, missing rows
and factors that are NULL, NaN, +-inf, -0.0 or +-1e16 beside small values,
split into random partitions and batches. Half the seeds draw from the dense
family (non-negative keys, dimensions that are outputs or summed or batch
dimensions), some of them large enough to cross the dense algorithm's block
edges. Every draw is made in the reference's order.

The SQL the fold stands for is evaluated here, independently of the kernels
and of oracle/: a hash join on the shared dimensions, GROUP BY the outputs
(NULL keys grouped together), SUM of the products, HAVING COUNT(*) > 0, and
the domain's LEFT JOIN with COALESCE to the default, with DataFusion's key
equality (FloatKeys::SignedZerosEqual: -0.0 and 0.0 one key, shown as 0.0).
The invariants (kernels_vs_sql.rs:17-37), in both product forms:

1. the same rows, as a multiset, keys compared by their bits;
2. values NULL where SQL gives NULL, NaN where it gives NaN, the same
   infinity, otherwise within 2(n-1)u sum|terms| (the FP64 form; the split
   form within that or its own bound, n terms each within (8 + 16(S+1))
   2^-8S of its row's and column's largest magnitudes);
3. other batchings give the same rows, bit for bit;
4. where the dense path runs with a domain, asking it to check that the
   domain's keys are unique declines exactly when two domain rows reach one
   group, and otherwise gives the same rows, bit for bit;
5. given exactly the bytes the kernels asked of an unlimited budget, the same
   rows by the same algorithm, bit for bit; given one byte fewer, a memory
   error.

Dictionary-encoded keys (NULL as a NULL dictionary value) run like the
plain columns of their values; the results carry them dictionary-encoded.
"""
import math
import struct

import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle

pytestmark = pytest.mark.gpu

SEED, CASES = 0x5EEDF01D, 400
U = 2.0 ** -53
FORMS = (K.Precision.FP64, K.Precision.SPLIT)
INT, POS, WIDE, TEXT, FLOAT, DICT = range(6)
LARGE = [[300, 7, 16], [3, 4, 5000], [3, 9000, 5]]
BATCHED = [520, 128, 4]
HOST = K.Host(K.FloatKeys.SIGNED_ZEROS_EQUAL)


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


# ---- keys and factors (kernels_vs_sql.rs:75-181) -----------------------------

def key_of(ty, i):
    if ty == INT:
        return i - 1
    if ty == POS:
        return i
    if ty == WIDE:
        return 1 << 63 if i == 0 else ((1 << 63) - 1 if i == 1 else i)
    if ty in (TEXT, DICT):
        return f"k{i}"
    return [0.0, -0.0, float("nan"), 2.5, -1.0][i % 5]


def arrow_type(ty):
    return {INT: pa.int64(), POS: pa.int64(), WIDE: pa.uint64(), TEXT: pa.string(), FLOAT: pa.float64(),
            DICT: pa.dictionary(pa.int32(), pa.string())}[ty]


def column(ty, keys):
    if ty != DICT:
        return pa.array(keys, type=arrow_type(ty))
    # NULLs as a NULL dictionary value (index 0), not a NULL index.
    dictionary, index = [None], {None: 0}
    idx = []
    for k in keys:
        if k not in index:
            index[k] = len(dictionary)
            dictionary.append(k)
        idx.append(index[k])
    return pa.DictionaryArray.from_arrays(pa.array(idx, type=pa.int32()), pa.array(dictionary, type=pa.string()))


def factor(rng, specials):
    r = rng.below(100)
    if 10 <= r <= 15 and not specials:
        r = 50
    if r <= 9:
        return None
    if r <= 12:
        return float("nan")
    if r <= 14:
        return float("inf")
    if r == 15:
        return float("-inf")
    if r <= 18:
        return -0.0
    if r <= 25:
        return 1e16 if rng.chance(0.5) else -1e16
    mantissa = (rng.next_u64() >> 11) / float(1 << 53) - 0.5
    return mantissa * 10.0 ** (rng.below(7) - 3)


class Rows:
    def __init__(self, present, duplicates, null_keys, specials, null_factors):
        self.present, self.duplicates, self.null_keys = present, duplicates, null_keys
        self.specials, self.null_factors = specials, null_factors


MESSY = Rows(0.75, True, True, True, True)


class Table:
    """Key columns (per dimension, as Python values, None for NULL), their
    types, and the factors."""

    def __init__(self, names, types, keys, values):
        self.names, self.types, self.keys, self.values = names, types, keys, values

    @property
    def rows(self):
        return len(self.values)

    def batch(self):
        cols = [column(t, k) for t, k in zip(self.types, self.keys)] + [pa.array(self.values, type=pa.float64())]
        return pa.RecordBatch.from_arrays(cols, names=list(self.names) + ["v"])

    def partitions(self, rng):
        """The rows in a random order, in random partitions of random
        batches, flattened in partition order (kernels_vs_sql.rs:194-219)."""
        n = self.rows
        order = list(range(n))
        for i in range(n - 1, 0, -1):
            j = rng.below(i + 1)
            order[i], order[j] = order[j], order[i]
        whole = self.batch().take(pa.array(order, type=pa.uint64()))
        parts = 1 + rng.below(3)
        out = [[] for _ in range(parts)]
        start = 0
        while start < n:
            ln = min(1 + rng.below(5), n - start)
            out[rng.below(parts)].append(whole.slice(start, ln))
            start += ln
        flat = [b for p in out for b in p]
        return whole.schema, flat or [whole.slice(0, 0)]


def table(rng, names, types, extents, how):
    keys = [[] for _ in names]
    values = []
    total = int(np.prod(extents)) if extents else 1
    for t0 in range(total):
        if not rng.chance(how.present):
            continue
        copies = 2 if how.duplicates and rng.chance(0.15) else 1
        t = t0
        tup = []
        for e, ty in zip(extents, types):
            i = t % e
            t //= e
            tup.append(None if (how.null_keys and rng.chance(0.08)) else key_of(ty, i))
        for _ in range(copies):
            for k, v in zip(keys, tup):
                k.append(v)
            f = factor(rng, how.specials)
            values.append(f if how.null_factors else (0.5 if f is None else f))
    return Table(names, types, keys, values)


# ---- cases (kernels_vs_sql.rs:330-558) ---------------------------------------

class Case:
    def __init__(self, n, types, equal, held, outputs, a, b, dims_a, dims_b, domain, domain_eq, missing, has_domain):
        self.n, self.types, self.equal, self.held, self.outputs = n, types, equal, held, outputs
        self.a, self.b, self.dims_a, self.dims_b = a, b, dims_a, dims_b
        self.domain, self.domain_eq, self.missing, self.has_domain = domain, domain_eq, missing, has_domain

    def fold(self, with_domain=True):
        def op(dims):
            return ir.Operand([(d, c) for c, d in enumerate(dims)], len(dims))

        dom = self.has_domain and with_domain
        eq = lambda e: ir.KeyEquality.EQUAL if e else ir.KeyEquality.NOT_DISTINCT  # noqa: E731
        outs = [ir.Output(d, ir.DomainKey(i, eq(self.domain_eq[i])) if dom else None)
                for i, d in enumerate(self.outputs)]
        return ir.Fold([ir.Dimension(eq(e)) for e in self.equal], [op(self.dims_a), op(self.dims_b)], outs,
                       domain=ir.Domain(tuple(range(len(self.outputs))), self.missing) if dom else None)

    def has_dictionary(self):
        return any(t == DICT for t in self.types)


def draw_case(rng, dense, large):
    dense = dense or large is not None
    n = 3 if large is not None else 1 + rng.below(4)
    types = []
    for _ in range(n):
        if dense:
            types.append(WIDE if (large is None and rng.chance(0.1)) else POS)
        else:
            types.append([INT, INT, TEXT, FLOAT, DICT][rng.below(5)])
    extents = list(large) if large is not None else [1 + rng.below(6 if dense else 4) for _ in range(n)]
    equal = [rng.chance(0.5) for _ in range(n)]
    held = []
    for d in range(n):
        r = [0, 2, 1][d] if large is not None else rng.below(3)
        held.append([r == 0 or r == 2, r == 1 or r == 2])
    batched = large == BATCHED
    outputs = []
    for d in range(n):
        if dense:
            keep = held[d] != [True, True] or batched or (large is None and rng.chance(0.3))
        else:
            keep = rng.chance(0.5)
        if keep:
            outputs.append(d)
    for i in range(len(outputs) - 1, 0, -1):
        j = rng.below(i + 1)
        outputs[i], outputs[j] = outputs[j], outputs[i]

    def how():
        if dense and large is not None:
            return Rows(1.0, False, False, rng.chance(0.5), False)
        if dense:
            present = 1.0 if rng.chance(0.6) else 0.75
            duplicates = rng.chance(0.2)
            specials = rng.chance(0.5)
            return Rows(present, duplicates, False, specials, True)
        return MESSY

    def side(s):
        mine = [d for d in range(n) if held[d][s]]
        t = table(rng, [f"k{d}" for d in mine], [types[d] for d in mine], [extents[d] for d in mine], how())
        return t, mine

    a, dims_a = side(0)
    b, dims_b = side(1)
    has_domain = rng.chance(0.5)
    dom = table(rng, [f"k{d}" for d in outputs], [types[d] for d in outputs], [extents[d] + 1 for d in outputs],
                MESSY) if has_domain else None
    domain_eq = [rng.chance(0.5) for _ in outputs] if has_domain else []
    missing = None
    if has_domain:
        m = rng.below(5 if dense else 3)
        missing = None if m == 0 else (2.5 if m == 1 else 0.0)
    return Case(n, types, equal, held, outputs, a, b, dims_a, dims_b, dom, domain_eq, missing, has_domain)


# ---- SQL's answer, evaluated here --------------------------------------------

def fbits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def canon(v):
    """A key as the host compares it (join and GROUP BY): NULL apart, floats
    by their bits with -0.0 as 0.0."""
    if v is None:
        return (0,)
    if isinstance(v, float):
        return (1, "f", fbits(0.0 if v == 0.0 else v))
    return (1, type(v).__name__, v)


def shown(v):
    """A key as printed, by its bits (-0.0 is not 0.0)."""
    if v is None:
        return (0,)
    if isinstance(v, float):
        return (1, "f", fbits(v))
    return (1, type(v).__name__, v)


class Group:
    __slots__ = ("key", "valued", "total", "count", "mag", "amax", "bmax")

    def __init__(self, key):
        self.key, self.valued, self.total, self.count, self.mag = key, False, 0.0, 0, 0.0
        self.amax = self.bmax = 0.0


def sql(case):
    """The fold's SQL: (shown keys, value or None, bound of the reference's
    sum, split-form scale n·max|a|·max|b|) per result row."""
    a, b = case.a, case.b
    shared = [d for d in range(case.n) if case.held[d] == [True, True]]
    ca = {d: c for c, d in enumerate(case.dims_a)}
    cb = {d: c for c, d in enumerate(case.dims_b)}

    def join_key(t, cols, r):
        k = []
        for d in shared:
            v = t.keys[cols[d]][r]
            if v is None and case.equal[d]:
                return None  # NULL joins nothing under '='
            k.append(canon(v))
        return tuple(k)

    by_key = {}
    for r in range(b.rows):
        k = join_key(b, cb, r)
        if k is not None:
            by_key.setdefault(k, []).append(r)

    def src(d):
        return (a, ca) if case.held[d][0] else (b, cb)

    # The split form scales each row of a (its own outputs and the batch
    # dimensions) and each column of b by their largest magnitudes.
    a_out = [d for d in case.outputs if case.held[d][0]]
    b_out = [d for d in case.outputs if case.held[d][1]]
    amax, bmax = {}, {}
    for t, cols, outs, m in ((a, ca, a_out, amax), (b, cb, b_out, bmax)):
        for r in range(t.rows):
            v = t.values[r]
            if v is None or not math.isfinite(v):
                continue
            k = tuple(canon(t.keys[cols[d]][r]) for d in outs)
            m[k] = max(m.get(k, 0.0), abs(v))

    groups = {}
    for ra in range(a.rows):
        k = join_key(a, ca, ra)
        if k is None:
            continue
        for rb in by_key.get(k, ()):
            vals = []
            for d in case.outputs:
                t, cols = (a, ca) if case.held[d][0] else (b, cb)
                vals.append(t.keys[cols[d]][ra if t is a else rb])
            gk = tuple(canon(v) for v in vals)
            g = groups.get(gk)
            if g is None:
                g = groups[gk] = Group(vals)
                g.amax = amax.get(tuple(canon(a.keys[ca[d]][ra]) for d in a_out), 0.0)
                g.bmax = bmax.get(tuple(canon(b.keys[cb[d]][rb]) for d in b_out), 0.0)
            g.count += 1
            x, y = a.values[ra], b.values[rb]
            if x is not None and y is not None:
                g.valued = True
                g.total += x * y
                g.mag += abs(x * y)

    def bound(g):
        return 2.0 * max(g.count - 1, 0) * U * g.mag

    def scale(g):
        return g.count * g.amax * g.bmax

    out = []
    if not case.has_domain:
        for g in groups.values():
            # A group of floats -0.0 and 0.0 shows as 0.0.
            key = tuple(shown(0.0 if (isinstance(v, float) and v == 0.0) else v) for v in g.key)
            out.append((key, g.total + 0.0 if g.valued else None, bound(g), scale(g)))
        return out
    d = case.domain
    for r in range(d.rows):
        lk = []
        for i in range(len(case.outputs)):
            v = d.keys[i][r]
            if v is None and case.domain_eq[i]:
                lk = None
                break
            lk.append(canon(v))
        g = groups.get(tuple(lk)) if lk is not None else None
        key = tuple(shown(d.keys[i][r]) for i in range(len(case.outputs)))
        if g is not None and g.valued:
            out.append((key, g.total + 0.0, bound(g), scale(g)))
        else:
            out.append((key, case.missing, 0.0, 0.0))
    return out


def rows_of(batches, nkeys):
    """Our result's rows: (shown keys, value or None), in order."""
    out = []
    for bt in batches:
        cols = []
        for c in range(nkeys):
            col = bt.column(c)
            if pa.types.is_dictionary(col.type):
                col = col.dictionary_decode()
            cols.append(col.to_pylist())
        vals = bt.column(nkeys).to_pylist()
        for r in range(bt.num_rows):
            out.append((tuple(shown(cols[c][r]) for c in range(nkeys)), vals[r]))
    return out


def bits_of(rows):
    nan = fbits(float("nan"))
    return [(k, None if v is None else (nan if v != v else fbits(v))) for k, v in rows]


def equivalent(ours, theirs, bound):
    if ours is None or theirs is None:
        return ours is None and theirs is None
    if ours != ours or theirs != theirs:
        return ours != ours and theirs != theirs
    if ours == theirs:
        return math.copysign(1.0, ours) == math.copysign(1.0, theirs)
    return math.isfinite(ours) and math.isfinite(theirs) and abs(ours - theirs) <= bound


# ---- the kernels' answers and the invariants (kernels_vs_sql.rs:652-1002) ----

class Limit(K.Budget):
    """A budget that counts what it gives, up to a limit."""

    def __init__(self, limit):
        self.given, self.limit = 0, limit

    def grow(self, n):
        if self.given + n > self.limit:
            return False
        self.given += n
        return True

    def shrink(self, n):
        self.given -= n


def batches_of(case, rng):
    """Each table's rows in a random order and batching (a, b, the domain)."""
    sa, ba = case.a.partitions(rng)
    sb, bb = case.b.partitions(rng)
    d = case.domain.partitions(rng) if case.has_domain else None
    return (sa, ba), (sb, bb), d


def fold_within(case, parts, form, budget=None, fold=None, dense_rows=None):
    (sa, ba), (sb, bb), d = parts
    fold = fold or case.fold()
    dom = K.Relation(d[0], d[1]) if (d is not None and fold.domain() is not None) else None
    o = K.Options(host=HOST, precision=form, budget=budget)
    if dense_rows is not None:
        o.domain_rows = dense_rows
        return K.fold_dense(fold, K.Relation(sa, ba), K.Relation(sb, bb), dom, options=o)
    return K.fold(fold, K.Relation(sa, ba), K.Relation(sb, bb), dom, options=o)


def run_fold(case, rng):
    parts = batches_of(case, rng)
    rng.below(8)  # threads: one device here
    return {f: fold_within(case, parts, f) for f in FORMS}


def check_budget(case, rng, form):
    parts = batches_of(case, rng)
    rng.below(8)
    free = Limit(float("inf"))
    base = fold_within(case, parts, form, free)
    asked = free.given
    assert free.given == asked
    exact = fold_within(case, parts, form, Limit(asked))
    assert exact.algorithm == base.algorithm, "given the bytes it asked for, another algorithm"
    assert bits_of(rows_of(exact.batches, len(case.outputs))) == bits_of(rows_of(base.batches, len(case.outputs))), \
        "given the bytes it asked for, other rows"
    if asked > 0:
        with pytest.raises(K.ArrowMemoryError):
            fold_within(case, parts, form, Limit(asked - 1))


def check_unique_domain(case, rng, form):
    """Invariant 4 for a case with a domain that the dense path computes;
    whether the checked path accepted."""
    parts = batches_of(case, rng)
    nk = len(case.outputs)
    rng.below(8)
    unchecked = fold_within(case, parts, form, dense_rows=K.DomainRows.ANY)
    assert unchecked is not None, "the dense path declined a fold it ran"
    rng.below(8)
    bare = fold_within(case, parts, form, fold=case.fold(with_domain=False), dense_rows=K.DomainRows.ANY)
    if bare is None:
        return False
    groups = {k for k, _ in rows_of(bare, nk)}
    seen, repeated = set(), False
    for k, _ in rows_of(unchecked, nk):
        if k in groups:
            if k in seen:
                repeated = True
            seen.add(k)
    rng.below(8)
    checked = fold_within(case, parts, form, dense_rows=K.DomainRows.UNIQUE_KEYS)
    if checked is None:
        return False
    assert not repeated, "the checked dense path accepted two domain rows with one group's keys"
    assert sorted(bits_of(rows_of(checked, nk))) == sorted(bits_of(rows_of(unchecked, nk))), \
        "the checked dense path changed the output"
    return True


def compare_with_sql(case, batches, form, theirs):
    nk = len(case.outputs)
    ours = rows_of(batches, nk)
    theirs = list(theirs)
    assert len(ours) == len(theirs), f"{len(ours)} rows, SQL has {len(theirs)}"
    ours.sort(key=lambda r: (r[0], r[1] is not None))
    theirs.sort(key=lambda r: (r[0], r[1] is not None))
    for (k, v), (wk, wv, bound, scale) in zip(ours, theirs):
        if form == K.Precision.SPLIT:
            bound += (8.0 + 16.0 * 7) * 2.0 ** -48 * scale
        assert k == wk and equivalent(v, wv, bound), f"row {k} = {v}, SQL's {wk} = {wv} within {bound:e}"


def large_of(seed):
    m = seed % 40
    if m in (1, 21):
        return LARGE[(seed // 20) % len(LARGE)]
    return BATCHED if m == 3 else None


def test_folds_match_sql():
    stats = dict(dense_family=0, dense_ran=0, batched_ran=0, large_batched_ran=0, unique_checked=0,
                 unique_accepted=0, with_dictionary=0, cases=0)
    failures = []
    for i in range(CASES):
        seed = SEED + i
        rng = Draws(seed, 0)
        dense = seed % 2 == 1
        large = large_of(seed)
        case = draw_case(rng, dense, large)
        stats["cases"] += 1
        nk = len(case.outputs)
        try:
            ours = run_fold(case, rng)
            stats["with_dictionary"] += case.has_dictionary()
            again = run_fold(case, rng)
            for f in FORMS:
                check_budget(case, rng, f)
            ran = ours[FORMS[0]].algorithm
            assert all(ours[f].algorithm == ran for f in FORMS)
            stats["dense_family"] += dense
            stats["dense_ran"] += ran == K.Algorithm.DENSE
            if large is not None:
                assert ran == K.Algorithm.DENSE, f"a large case of shape {large} ran {ran}"
            batched = any(case.held[d] == [True, True] for d in case.outputs)
            stats["batched_ran"] += batched and ran == K.Algorithm.DENSE
            stats["large_batched_ran"] += large == BATCHED and ran == K.Algorithm.DENSE
            if ran == K.Algorithm.DENSE and case.has_domain:
                stats["unique_checked"] += 1
                stats["unique_accepted"] += check_unique_domain(case, rng, FORMS[1])
            theirs = sql(case)
            for f in FORMS:
                assert sorted(bits_of(rows_of(ours[f].batches, nk))) == sorted(bits_of(rows_of(again[f].batches, nk))), \
                    f"two arrival orders gave different outputs ({f.name})"
                compare_with_sql(case, ours[f].batches, f, theirs)
        except AssertionError as e:
            failures.append(f"seed {seed}: {e}")
    print(stats)
    assert not failures, "\n".join(failures[:20])
    assert stats["dense_ran"] * 4 >= stats["dense_family"], stats
    assert stats["batched_ran"] > 0 and stats["large_batched_ran"] > 0, stats
