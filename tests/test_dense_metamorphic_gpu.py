"""The reference's metamorphic properties of the dense fold
(crates/einfold-kernels/tests/dense_metamorphic.rs), on the B200 path.

Cases are drawn as that test draws them (dense_metamorphic.rs:128-349), from
its default seed on, with the SplitMix64 stream of einfold's test kit: the
flattened extents of each role at and around the reference's block edges
(256 output rows, 2,048 output columns, 4,096 positions of z, the switch at
4,096 output cells), factored into one or two dimensions; factors with
NULL, NaN, inf, -0.0 and +-1e16; half the cases with a domain (keys one past
each extent, repeated rows, NULL keys, either equality); and a few sparse
cases. Every draw is made in the reference's order, so a seed gives the
reference's case, batching and permutations.

Each case runs through einfold_fold / einfold_fold_dense in both product
forms, with the same batches, and checks the invariants
(dense_metamorphic.rs:693-925):

- [oracle] the result is a nested-loop evaluation of SQL's semantics: the
  same groups or domain rows, NULL where SQL gives NULL, NaN where it gives
  NaN, otherwise within 2(n-1)u sum|terms| (the FP64 form, which adds in the
  reference's order); the split form within that or its own bound, K terms
  each within (8 + 16(S+1)) 2^-8S of the product of its row's and column's
  largest magnitudes;
- [sparse] a sparse case runs the discrimination algorithm;
- [threads] other batching gives the same bits;
- [scale] doubling and negating a's factors doubles and negates every
  result, bit for bit; in the split form negating holds within its bound
  only: balanced base-256 digits lie in [-128, 127], so -W's digits are not
  the negated digits of W where one of them is -128, and the digit pairs the
  split product leaves out then differ (doubling moves only the exponent);
- [relabel] permuting output keys permutes the result's keys and keeps
  every value's bits;
- [key-type] keys as Int32, Int16 or UInt32 give the same bits;
- [domain] each domain row gets its group's bits from the fold without a
  domain, or the default;
- [unique] with the domain's keys checked, the dense algorithm declines
  exactly when two in-range domain rows share a cell, else the same bits;
- [discriminate] a row of b that joins nothing moves the fold to the
  discrimination algorithm, with the oracle's rows;
- [duplicates] a repeated row moves it there too, summed twice;
- [swap] swapping the operands gives the oracle's rows.

The oracle here is independent of the kernels and of oracle/: numpy over
dense layers of the relations' rows.
"""
import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle

pytestmark = pytest.mark.gpu

NULL_KEY = -(1 << 63)
# The dense algorithm's block sizes (dense.rs) and the edges the cases aim at.
XB, YB, ZB, FEW_CELLS = 256, 2048, 4096, 4096
X_EDGES = [1, 2, 3, 64, XB - 1, XB, XB + 1, 2 * XB, 2 * XB + 1]
Y_EDGES = [1, 2, 5, YB - 1, YB, YB + 1, 2 * YB + 1]
Z_EDGES = [1, 2, 3, 16, ZB - 1, ZB, ZB + 1]
WORK_CAP = 3_000_000  # the oracle's work cap of a debug build of the reference's test
SEED, CASES = 0x000B10C5, 60
U = 2.0 ** -53
FORMS = (K.Precision.FP64, K.Precision.SPLIT)


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


class Rel:
    def __init__(self, dims, keys, values):
        self.dims, self.keys, self.values = list(dims), keys, values  # keys: rows of ints; values: float or None

    def copy(self):
        return Rel(self.dims, [list(k) for k in self.keys], list(self.values))


class Dom:
    def __init__(self, rel, missing, equality):
        self.rel, self.missing, self.equality = rel, missing, equality


class Case:
    def __init__(self, xs, zs, ys, outputs, extent, a, b, domain, sparse):
        self.xs, self.zs, self.ys, self.outputs, self.extent = xs, zs, ys, outputs, extent
        self.a, self.b, self.domain, self.sparse = a, b, domain, sparse

    def copy(self):
        d = None if self.domain is None else Dom(self.domain.rel.copy(), self.domain.missing, self.domain.equality)
        return Case(self.xs, self.zs, self.ys, self.outputs, self.extent, self.a.copy(), self.b.copy(), d,
                    self.sparse)

    def cells(self, dims):
        return int(np.prod([self.extent[d] for d in dims])) if dims else 1


# ---- drawing cases (dense_metamorphic.rs:128-349) ----------------------------

def value(rng, specials):
    c = rng.below(100)
    if c <= 4:
        return None
    if 5 <= c <= 6 and specials:
        return float("nan")
    if c == 7 and specials:
        return float("inf")
    if 8 <= c <= 10:
        return -0.0
    if 11 <= c <= 16:
        return 1e16 if rng.chance(0.5) else -1e16
    return ((rng.next_u64() >> 11) / float(1 << 53) - 0.5) * 8.0


def factor(rng, t, empty):
    if t == 1 and empty and rng.chance(0.5):
        return []
    divisors = [d for d in range(2, t) if t % d == 0]
    if divisors and rng.chance(0.5):
        d = rng.pick(divisors)
        return [d, t // d]
    return [t]


def rel(rng, dims, extent, present, specials):
    total = int(np.prod([extent[d] for d in dims])) if dims else 1
    keys, values = [], []
    for t0 in range(total):
        if t0 + 1 < total and not rng.chance(present):
            continue
        t, k = t0, [0] * len(dims)
        for slot in range(len(dims) - 1, -1, -1):
            e = extent[dims[slot]]
            k[slot] = t % e
            t //= e
        keys.append(k)
        values.append(value(rng, specials))
    return Rel(dims, keys, values)


def domain(rng, outputs, extent):
    ext = [e + 1 for e in extent]
    d = rel(rng, outputs, ext, 0.6, False)
    if rng.chance(0.6):
        n = len(d.keys)
        extra = [rng.below(n) for _ in range(n // 10 + 1)]
        for i in extra:
            d.keys.append(list(d.keys[i]))
            d.values.append(None)
    if rng.chance(0.3):
        for k in d.keys:
            for s in range(len(k)):
                if rng.chance(0.1):
                    k[s] = NULL_KEY
    equality = [ir.KeyEquality.EQUAL if rng.chance(0.5) else ir.KeyEquality.NOT_DISTINCT for _ in outputs]
    missing = [None, 0.0, 2.5][rng.below(3)]
    return Dom(d, missing, equality)


def sparse_case(rng):
    extent = [1 + rng.below(5), 1_000_000, 1 + rng.below(5)]
    z_keys = [rng.below(1_000_000) for _ in range(300)]

    def over(dims, other):
        keys, values = [], []
        for z in z_keys:
            if rng.chance(0.8):
                o = rng.below(extent[other])
                keys.append([z, o] if dims[0] == 1 else [o, z])
                values.append(value(rng, False))
        return Rel(dims, keys, values)

    a = over([0, 1], 0)
    b = over([1, 2], 2)
    outputs = [0, 2]
    dom = domain(rng, outputs, extent) if rng.chance(0.5) else None
    return Case([0], [1], [2], outputs, extent, a, b, dom, True)


def draw_case(rng):
    if rng.chance(0.06):
        return sparse_case(rng)
    near = lambda edge: edge - 1 + rng.below(3)  # noqa: E731
    small = lambda: 1 + rng.below(6)  # noqa: E731
    kind = rng.below(10)
    if kind <= 2:
        p = near(FEW_CELLS)
        nx = rng.pick([d for d in range(1, p + 1) if p % d == 0])
        nx, ny, nz = nx, p // nx, rng.pick(Z_EDGES[:4])
    elif kind <= 4:
        nx = near(XB)
        ny = 17 + rng.below(24)
        nz = small()
    elif kind <= 6:
        nx = 2 + rng.below(5)
        ny = near(YB)
        nz = small()
    elif kind == 7:
        nx = small()
        ny = small()
        nz = near(ZB)
    else:
        def pick_edge(edges):
            return 1 + rng.below(6) if rng.chance(0.25) else rng.pick(edges)

        nx = pick_edge(X_EDGES)
        ny = pick_edge(Y_EDGES)
        nz = pick_edge(Z_EDGES)

    def fits(z):
        return nx * z <= 300_000 and z * ny <= 300_000 and nx * ny <= 600_000 and nx * z * ny <= WORK_CAP

    if not fits(nz):
        nz = 1 + rng.below(3)
    if not fits(nz):
        return None
    fx, fz, fy = factor(rng, nx, True), factor(rng, nz, False), factor(rng, ny, True)
    extent = []

    def role(sizes):
        out = []
        for e in sizes:
            extent.append(e)
            out.append(len(extent) - 1)
        return out

    xs, zs, ys = role(fx), role(fz), role(fy)
    outputs = xs + ys
    for i in range(len(outputs) - 1, 0, -1):
        j = rng.below(i + 1)
        outputs[i], outputs[j] = outputs[j], outputs[i]
    specials = rng.chance(0.2)
    pa_ = 1.0 if rng.chance(0.5) else 0.7
    pb_ = 1.0 if rng.chance(0.85) else 0.9
    a = rel(rng, xs + zs, extent, pa_, specials)
    b = rel(rng, zs + ys, extent, pb_, specials)
    if rng.chance(0.7):
        b.values = [0.25 if v is None else v for v in b.values]
    dom = domain(rng, outputs, extent) if rng.chance(0.5) else None
    return Case(xs, zs, ys, outputs, extent, a, b, dom, False)


# ---- running a case through the library --------------------------------------

def batch_of(r, ty):
    n = len(r.keys)
    keys = np.array(r.keys, dtype=np.int64).reshape(n, len(r.dims))
    cols = []
    for c in range(len(r.dims)):
        k = keys[:, c]
        null = k == NULL_KEY
        cols.append(pa.array(np.where(null, 0, k), type=pa.int64(), mask=null).cast(ty))
    v = np.array([0.0 if x is None else x for x in r.values], dtype=np.float64)
    vnull = np.array([x is None for x in r.values], dtype=bool)
    cols.append(pa.array(v, type=pa.float64(), mask=vnull))
    schema = pa.schema([pa.field(f"k{i}", ty) for i in range(len(r.dims))] + [pa.field("v", pa.float64())])
    return schema, pa.RecordBatch.from_arrays(cols, schema=schema)


def split(rng, b):
    n = b.num_rows
    order = list(range(n))
    for i in range(n - 1, 0, -1):
        j = rng.below(i + 1)
        order[i], order[j] = order[j], order[i]
    taken = b.take(pa.array(order, type=pa.uint32()))
    out, at = [], 0
    while at < n:
        ln = min(rng.below(n // 3 + 2), n - at)
        out.append(taken.slice(at, ln))
        at += ln
    return out


def fold_of(case, swapped, with_domain):
    def op(r):
        return ir.Operand([(d, c) for c, d in enumerate(r.dims)], len(r.dims))

    ops = [op(case.b), op(case.a)] if swapped else [op(case.a), op(case.b)]
    dom = case.domain if with_domain else None
    outs = [ir.Output(d, ir.DomainKey(i, dom.equality[i]) if dom else None) for i, d in enumerate(case.outputs)]
    return ir.Fold([ir.EQ] * len(case.extent), ops, outs,
                   domain=ir.Domain(tuple(range(len(dom.rel.dims))), dom.missing) if dom else None)


class Run:
    def __init__(self, algorithm, batches):
        self.algorithm, self.batches = algorithm, batches


def run(case, rng, ty, swapped, with_domain, mode):
    """The case's fold in each product form, on one batching: mode "best"
    (einfold_fold), or a DomainRows for einfold_fold_dense (None where it
    declines). The thread count is drawn as the reference draws it."""
    rng.below(8)  # threads: one device here
    f = fold_of(case, swapped, with_domain)
    first, second = (case.b, case.a) if swapped else (case.a, case.b)
    sa, ba = batch_of(first, ty)
    sb, bb = batch_of(second, ty)
    dom = batch_of(case.domain.rel, ty) if (case.domain is not None and with_domain) else None
    ba, bb = split(rng, ba), split(rng, bb)
    bd = split(rng, dom[1]) if dom else None
    d = K.Relation(dom[0], bd) if dom else None
    out = {}
    for form in FORMS:
        o = K.Options(host=K.Host(K.FloatKeys.SIGNED_ZEROS_EQUAL), precision=form)
        if mode == "best":
            got = K.fold(f, K.Relation(sa, ba), K.Relation(sb, bb), d, options=o)
            out[form] = Run(got.algorithm, got.batches)
        else:
            o.domain_rows = mode
            got = K.fold_dense(f, K.Relation(sa, ba), K.Relation(sb, bb), d, options=o)
            out[form] = None if got is None else Run(K.Algorithm.DENSE, got)
    return out


def rows(batches, nkeys):
    """A result's rows as (keys [n, k] int64 with NULL_KEY, values, NULL
    mask), sorted by keys then value bits."""
    ks, vs, ns = [], [], []
    for b in batches:
        ks.append(np.stack([np.where(b.column(c).is_null().to_numpy(zero_copy_only=False), NULL_KEY,
                                     b.column(c).cast(pa.int64()).fill_null(0).to_numpy(zero_copy_only=False))
                            for c in range(nkeys)], 1) if nkeys else np.zeros((b.num_rows, 0), np.int64))
        v = b.column(nkeys)
        ns.append(v.is_null().to_numpy(zero_copy_only=False))
        vs.append(v.fill_null(0.0).to_numpy(zero_copy_only=False).astype(np.float64))
    k = np.concatenate(ks) if ks else np.zeros((0, nkeys), np.int64)
    v = np.concatenate(vs) if vs else np.zeros(0)
    n = np.concatenate(ns).astype(bool) if ns else np.zeros(0, bool)
    return sort_rows(k, v, n)


def value_bits(v, null):
    b = v.view(np.uint64).copy()
    b[np.isnan(v)] = np.float64("nan").view(np.uint64)
    b[null] = 0
    return b


def sort_rows(k, v, n):
    order = np.lexsort([value_bits(v, n), n] + [k[:, c] for c in range(k.shape[1] - 1, -1, -1)])
    return k[order], v[order], n[order]


def same_bits(x, y):
    return (len(x[0]) == len(y[0]) and np.array_equal(x[0], y[0]) and np.array_equal(x[2], y[2])
            and np.array_equal(value_bits(x[1], x[2]), value_bits(y[1], y[2])))


# ---- the oracle: SQL's groups over dense layers of the rows ----------------

def uniq(t):
    """The distinct key tuples of t's rows, and each row's index among them
    (one empty tuple when t has no columns)."""
    if t.shape[1] == 0:
        return np.zeros((1, 0), np.int64), np.zeros(len(t), np.int64)
    u, i = np.unique(t, axis=0, return_inverse=True)
    return u, i.reshape(-1)


def groups_of(case, split_form):
    """Each group's keys (in output order), value (None: NULL), and bound."""
    a, b = case.a, case.b
    ka = np.array(a.keys, dtype=np.int64).reshape(len(a.keys), len(a.dims))
    kb = np.array(b.keys, dtype=np.int64).reshape(len(b.keys), len(b.dims))
    col_a = {d: c for c, d in enumerate(a.dims)}
    col_b = {d: c for c, d in enumerate(b.dims)}
    za = ka[:, [col_a[d] for d in case.zs]]
    zb = kb[:, [col_b[d] for d in case.zs]]
    xa = ka[:, [col_a[d] for d in case.xs]]
    yb = kb[:, [col_b[d] for d in case.ys]]
    zu, zi = np.unique(np.concatenate([za, zb]), axis=0, return_inverse=True)
    zi = zi.reshape(-1)
    zia, zib = zi[:len(za)], zi[len(za):]
    xu, xia = uniq(xa)
    yu, yib = uniq(yb)
    nx, ny, nz = len(xu), len(yu), len(zu)
    va = np.array([np.nan if x is None else x for x in a.values], dtype=np.float64)
    vb = np.array([np.nan if x is None else x for x in b.values], dtype=np.float64)
    na = np.array([x is None for x in a.values], dtype=bool)
    nb = np.array([x is None for x in b.values], dtype=bool)

    def layers(p, q, vals, nulls, shape):
        # Rows at the same cell go to successive layers, so each layer is a
        # dense matrix; a pair of layers joins as SQL joins their rows.
        cell = p * shape[1] + q
        order = np.argsort(cell, kind="stable")
        c_sorted = cell[order]
        first = np.r_[True, c_sorted[1:] != c_sorted[:-1]]
        run_start = np.maximum.accumulate(np.where(first, np.arange(len(c_sorted)), 0))
        occ = np.empty(len(cell), np.int64)
        occ[order] = np.arange(len(c_sorted)) - run_start
        out = []
        for lvl in range(int(occ.max()) + 1 if len(occ) else 0):
            m = occ == lvl
            present = np.zeros(shape, bool)
            valued = np.zeros(shape, bool)
            x = np.zeros(shape)
            present[p[m], q[m]] = True
            valued[p[m], q[m]] = ~nulls[m]
            x[p[m], q[m]] = np.where(nulls[m], 0.0, vals[m])
            out.append((present, valued, x))
        return out

    la = layers(xia, zia, va, na, (nx, nz))
    lb = layers(zib, yib, vb, nb, (nz, ny))
    exists = np.zeros((nx, ny), bool)
    valued = np.zeros((nx, ny), bool)
    total = np.zeros((nx, ny))
    terms = np.zeros((nx, ny))
    mag = np.zeros((nx, ny))
    for pa_, va_, xa_ in la:
        for pb_, vb_, xb_ in lb:
            exists |= (pa_.astype(np.int64) @ pb_.astype(np.int64)) > 0
            both = va_.astype(np.int64) @ vb_.astype(np.int64)
            valued |= both > 0
            terms += both
            step = max(1, 2_000_000 // max(1, nz * ny))
            for x0 in range(0, nx, step):
                sl = slice(x0, x0 + step)
                m = va_[sl][:, :, None] & vb_[None]
                with np.errstate(invalid="ignore", over="ignore"):
                    prod = np.where(m, xa_[sl][:, :, None] * xb_[None], 0.0)
                    total[sl] = total[sl] + prod.sum(axis=1)
                    mag[sl] += np.abs(prod).sum(axis=1)
    total = total + 0.0  # SQL's sum starts at +0.0
    with np.errstate(invalid="ignore"):
        bound = 2.0 * np.maximum(terms - 1.0, 0.0) * U * mag
    if split_form:
        # Rows' and columns' largest finite magnitudes over the valued factors.
        fa = np.zeros((nx, nz))
        fb = np.zeros((nz, ny))
        for _, va_, xa_ in la:
            fa = np.maximum(fa, np.where(va_ & np.isfinite(xa_), np.abs(xa_), 0.0))
        for _, vb_, xb_ in lb:
            fb = np.maximum(fb, np.where(vb_ & np.isfinite(xb_), np.abs(xb_), 0.0))
        kk = max(1, nz) * len(la) * len(lb)
        bound = bound + kk * (8.0 + 16.0 * 7) * 2.0 ** -48 * np.outer(fa.max(1), fb.max(0))
    gx, gy = np.nonzero(exists)
    keys = np.zeros((len(gx), len(case.outputs)), np.int64)
    for s, d in enumerate(case.outputs):
        if d in case.xs:
            keys[:, s] = xu[gx, case.xs.index(d)]
        else:
            keys[:, s] = yu[gy, case.ys.index(d)]
    return keys, total[gx, gy], ~valued[gx, gy], bound[gx, gy]


def expected(case, with_domain, split_form):
    keys, vals, nulls, bound = groups_of(case, split_form)
    dom = case.domain if with_domain else None
    if dom is not None:
        index = {tuple(k): i for i, k in enumerate(keys.tolist())}
        n = len(dom.rel.keys)
        dk = np.array(dom.rel.keys, dtype=np.int64).reshape(n, len(case.outputs))
        v = np.zeros(n)
        nl = np.zeros(n, bool)
        bd = np.zeros(n)
        for r, k in enumerate(dom.rel.keys):
            i = index.get(tuple(k)) if NULL_KEY not in k else None
            if i is not None and not nulls[i]:
                v[r], bd[r] = vals[i], bound[i]
            else:
                v[r] = 0.0 if dom.missing is None else dom.missing
                nl[r] = dom.missing is None
        keys, vals, nulls, bound = dk, v, nl, bd
    order = np.lexsort([value_bits(vals, nulls), nulls] + [keys[:, c] for c in range(keys.shape[1] - 1, -1, -1)])
    return keys[order], vals[order], nulls[order], bound[order]


def check_matches(tag, ours, want):
    k, v, n = ours
    wk, wv, wn, wb = want
    assert len(k) == len(wk), f"[{tag}] {len(k)} rows, the oracle has {len(wk)}"
    assert np.array_equal(k, wk), f"[{tag}] keys differ"
    assert np.array_equal(n, wn), f"[{tag}] NULLs differ"
    live = ~n
    x, y, bd = v[live], wv[live], wb[live]
    nan = np.isnan(x) | np.isnan(y)
    assert np.array_equal(np.isnan(x), np.isnan(y)), f"[{tag}] NaNs differ"
    eq = (x == y) & ~nan
    assert np.array_equal(np.signbit(x[eq]), np.signbit(y[eq])), f"[{tag}] signed zeros differ"
    rest = ~nan & ~eq
    ok = np.isfinite(x[rest]) & np.isfinite(y[rest]) & (np.abs(x[rest] - y[rest]) <= bd[rest])
    assert ok.all(), f"[{tag}] {int((~ok).sum())} values outside the bound; first {x[rest][~ok][:3]} vs {y[rest][~ok][:3]}"


def map_a(case, f):
    c = case.copy()
    c.a.values = [None if v is None else f(v) for v in c.a.values]
    return c


# ---- the invariants (dense_metamorphic.rs:693-925) --------------------------

def check(seed, stats):
    rng = Draws(seed, 0)
    stats["seeds"] += 1
    case = draw_case(rng)
    if case is None:
        stats["skipped"] += 1
        return
    stats["cases"] += 1
    nk = len(case.outputs)
    i64 = pa.int64()
    first = run(case, rng, i64, False, True, "best")
    ours = {f: rows(first[f].batches, nk) for f in FORMS}
    want = {f: expected(case, True, f == K.Precision.SPLIT) for f in FORMS}
    for f in FORMS:
        check_matches(f"oracle {f.name}", ours[f], want[f])
    if case.domain is not None and any(NULL_KEY in k for k in case.domain.rel.keys):
        stats["null_domain_keys"] += 1
    if case.sparse:
        stats["sparse"] += 1
        assert all(first[f].algorithm == K.Algorithm.DISCRIMINATE for f in FORMS), "[sparse] dense ran"
        return
    alg = first[FORMS[0]].algorithm
    assert all(first[f].algorithm == alg for f in FORMS)
    dense = alg == K.Algorithm.DENSE
    if dense:
        stats["dense"] += 1
        nx, nz, ny = case.cells(case.xs), case.cells(case.zs), case.cells(case.ys)
        blocked = nx * ny >= FEW_CELLS
        stats["blocked" if blocked else "z_blocked"] += 1
        near = lambda n, e: e - 1 <= n <= e + 1  # noqa: E731
        stats["at_switch"] += near(nx * ny, FEW_CELLS)
        stats["at_row_edge"] += blocked and near(nx, XB)
        stats["at_column_edge"] += blocked and near(ny, YB)
        stats["at_z_edge"] += (not blocked) and near(nz, ZB)

    # [threads]
    again = run(case, rng, i64, False, True, "best")
    for f in FORMS:
        assert same_bits(rows(again[f].batches, nk), ours[f]), f"[threads {f.name}] other batches changed the bits"

    # [scale]
    base = run(case, rng, i64, False, False, "best")
    base_rows = {f: rows(base[f].batches, nk) for f in FORMS}
    for tag, fn, vec in (("doubling", lambda v: v * 2.0, lambda v: v * 2.0), ("negating", lambda v: -v, np.negative)):
        mapped_case = map_a(case, fn)
        mapped = run(mapped_case, rng, i64, False, False, "best")
        for f in FORMS:
            if mapped[f].algorithm != base[f].algorithm:
                continue
            if f == K.Precision.SPLIT and tag == "negating" and mapped[f].algorithm == K.Algorithm.DENSE:
                check_matches("scale negating SPLIT", rows(mapped[f].batches, nk), expected(mapped_case, False, True))
                continue
            k, v, n = base_rows[f]
            wv = vec(v)
            zero = lambda x: np.where(x == 0.0, 0.0, x)  # noqa: E731
            got = rows(mapped[f].batches, nk)
            w = sort_rows(k, zero(wv), n)
            g = sort_rows(got[0], zero(got[1]), got[2])
            assert same_bits(g, w), f"[scale {f.name}] {tag} a's factors didn't {tag} the results exactly"

    # [relabel]
    perms = {}
    for d in case.xs + case.ys:
        p = list(range(case.extent[d]))
        for i in range(len(p) - 1, 0, -1):
            j = rng.below(i + 1)
            p[i], p[j] = p[j], p[i]
        perms[d] = p

    def apply(d, k):
        p = perms.get(d)
        return p[k] if p is not None and 0 <= k < len(p) else k

    def relabel(r):
        r.keys = [[apply(d, k) for d, k in zip(r.dims, row)] for row in r.keys]

    relabeled = case.copy()
    relabel(relabeled.a)
    relabel(relabeled.b)
    if relabeled.domain is not None:
        relabel(relabeled.domain.rel)
    r = run(relabeled, rng, i64, False, True, "best")
    for f in FORMS:
        if r[f].algorithm == first[f].algorithm:
            k, v, n = ours[f]
            k2 = k.copy()
            for s, d in enumerate(case.outputs):
                if d in perms:
                    p = np.array(perms[d], dtype=np.int64)
                    col = k[:, s]
                    inr = (col >= 0) & (col < len(p))
                    k2[inr, s] = p[col[inr]]
            assert same_bits(rows(r[f].batches, nk), sort_rows(k2, v, n)), \
                f"[relabel {f.name}] permuting output keys changed a value's bits"

    # [key-type]
    ty = [pa.int32(), pa.int16(), pa.uint32()][rng.below(3)]

    def fits(rel_):
        return all(k == NULL_KEY or 0 <= k < 32_000 for row in rel_.keys for k in row)

    if fits(case.a) and fits(case.b) and (case.domain is None or fits(case.domain.rel)):
        narrow = run(case, rng, ty, False, True, "best")
        for f in FORMS:
            if narrow[f].algorithm == first[f].algorithm:
                assert same_bits(rows(narrow[f].batches, nk), ours[f]), f"[key-type {f.name}] {ty} keys changed the bits"

    # [domain]
    if case.domain is not None:
        for f in FORMS:
            if base[f].algorithm != first[f].algorithm:
                continue
            bk, bv, bn = base_rows[f]
            groups = {tuple(k): (None if nl else val) for k, val, nl in zip(bk.tolist(), bv.tolist(), bn.tolist())}
            missing = case.domain.missing
            k, v, n = ours[f]
            for kk, vv, nn in zip(k.tolist(), v.tolist(), n.tolist()):
                g = groups.get(tuple(kk))
                expect = g if g is not None else missing
                got = None if nn else vv
                same = (expect is None and got is None) or (
                    expect is not None and got is not None and
                    np.float64(expect).view(np.uint64) == np.float64(got).view(np.uint64))
                assert same, f"[domain {f.name}] row {kk} = {got}, its group without a domain gives {expect}"

    # [unique]
    if case.domain is not None and dense:
        def in_range(k):
            return all(x != NULL_KEY and 0 <= x < case.extent[d] for x, d in zip(k, case.outputs))

        seen, repeated = set(), False
        for k in case.domain.rel.keys:
            if in_range(k):
                t = tuple(k)
                if t in seen:
                    repeated = True
                    break
                seen.add(t)
        unchecked = run(case, rng, i64, False, True, K.DomainRows.ANY)
        checked = run(case, rng, i64, False, True, K.DomainRows.UNIQUE_KEYS)
        for f in FORMS:
            u, c = unchecked[f], checked[f]
            assert u is not None, f"[unique {f.name}] the dense algorithm declined a fold it ran"
            if c is not None:
                assert not repeated, f"[unique {f.name}] accepted two domain rows that share a cell"
                stats["unique_accepted"] += f == FORMS[0]
                assert same_bits(rows(u.batches, nk), rows(c.batches, nk)), \
                    f"[unique {f.name}] checking the domain's keys changed the bits"
            else:
                assert repeated, f"[unique {f.name}] declined a domain whose rows have distinct cells"
                stats["unique_declined"] += f == FORMS[0]

    # [discriminate]
    extra = case.copy()
    extra.b.keys.append([-1] * len(extra.b.dims))
    extra.b.values.append(1.0)
    disc = run(extra, rng, i64, False, True, "best")
    for f in FORMS:
        assert disc[f].algorithm == K.Algorithm.DISCRIMINATE, \
            "[discriminate] a negative key didn't move the fold to the discrimination algorithm"
        check_matches(f"discriminate {f.name}", rows(disc[f].batches, nk), want[K.Precision.FP64])

    # [duplicates]
    if dense:
        dup = case.copy()
        side = dup.a if rng.chance(0.5) else dup.b
        r_ = rng.below(len(side.keys))
        side.keys.append(list(side.keys[r_]))
        side.values.append(0.5)
        ran = run(dup, rng, i64, False, True, "best")
        want_dup = expected(dup, True, False)
        for f in FORMS:
            assert ran[f].algorithm == K.Algorithm.DISCRIMINATE, "[duplicates] a repeated key tuple stayed dense"
            check_matches(f"duplicates {f.name}", rows(ran[f].batches, nk), want_dup)
        stats["duplicates"] += 1

    # [swap]
    if case.domain is None:
        sw = run(case, rng, i64, True, True, "best")
        for f in FORMS:
            check_matches(f"swap {f.name}", rows(sw[f].batches, nk), want[f])


def test_dense_metamorphic_properties():
    stats = {k: 0 for k in ("seeds", "skipped", "cases", "dense", "blocked", "z_blocked", "at_switch", "at_row_edge",
                            "at_column_edge", "at_z_edge", "unique_accepted", "unique_declined", "null_domain_keys",
                            "duplicates", "sparse")}
    failures = []
    seed = SEED
    while stats["cases"] < CASES and stats["seeds"] < 4 * CASES:
        try:
            check(seed, stats)
        except AssertionError as e:
            failures.append(f"seed {seed}: {e}")
        seed += 1
    print(stats)
    assert not failures, "\n".join(failures)
    assert stats["cases"] >= CASES, stats
    reached = [("the dense algorithm ran in a quarter of cases", stats["dense"] * 4 >= stats["cases"]),
               ("the output was blocked", stats["blocked"] > 0), ("z was blocked", stats["z_blocked"] > 0),
               ("nx*ny was at the switch", stats["at_switch"] > 0), ("nx was at a row edge", stats["at_row_edge"] > 0),
               ("ny was at a column edge", stats["at_column_edge"] > 0), ("nz was at a z edge", stats["at_z_edge"] > 0),
               ("the unique check accepted", stats["unique_accepted"] > 0),
               ("the unique check declined", stats["unique_declined"] > 0),
               ("a domain had NULL keys", stats["null_domain_keys"] > 0),
               ("a duplicate moved to discrimination", stats["duplicates"] > 0), ("a sparse case ran", stats["sparse"] > 0)]
    for what, ok in reached:
        assert ok, f"coverage: expected that {what}: {stats}"
