"""The oracle pinned to the reference's own known answers, on the CPU. The
SplitMix64 outputs of crates/einfold-testkit/src/rng.rs:66-78, the tile
counts of crates/einfold-kernels/tests/pipeline_vs_sql.rs:731-760, the
Bounds cases of crates/einfold-kernels/src/fused.rs:1116-1177, the long
shared prefix of discriminate.rs:663-683 and the property tests' seeds and
case counts are read from tests/golden/reference_facts.json, which
tests/golden/make_golden.py extracts from the reference's sources. Also: the
signed zero keys of keys.rs:83-93, the rounding bound and repeatability of
the dense product (kernels_vs_sql.rs:21-23, gemm.rs:52-89), the row-format
order of decimal keys, and the row-expression restatement held to SQL on the
reference's expression cases (expression_vs_sql.rs)."""
import math

import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir
from oracle import oracle
from tests import pipelines as P
from tests.tables import complete, matmul_fold, reference_facts, rows_of

GE, GT, LE, LT = (ir.Comparison.GREATER_OR_EQUAL, ir.Comparison.GREATER, ir.Comparison.LESS_OR_EQUAL,
                  ir.Comparison.LESS)
COMPARISONS = {"ge": GE, "gt": GT, "le": LE, "lt": LT}

FACTS = reference_facts()


def _f64(x):
    return float(x) if isinstance(x, str) else x


def test_splitmix64_seed_zero_gives_the_reference_outputs():
    want = FACTS["splitmix64_seed0"]["outputs"]
    assert len(want) == 4
    rng = oracle.Rng.seeded(0, 0)
    assert [rng.next_u64() for _ in range(4)] == want
    # The vectorised stream is the same stream.
    assert list(oracle.Rng.seeded(0, 0).u64s(4)) == want
    a, b = oracle.Rng.seeded(5, 1), oracle.Rng.seeded(5, 2)
    assert a.next_u64() != b.next_u64()


def _tiles(l, nb=None, conditions=()):
    r = P.run_oracle(P.attention(l, nb=nb, conditions=conditions))
    vals = rows_of(r.batches).column(rows_of(r.batches).num_columns - 1).to_numpy()
    assert len(vals) == l * (nb or 1)
    assert np.all(np.abs(vals - 1.0) < 1e-12)  # every average of v = 1 is 1
    return r.tiles_visited, r.tiles


@pytest.mark.parametrize("case", FACTS["tile_counts"], ids=lambda c: c["test"])
def test_masked_pipelines_visit_the_reference_tile_counts(case):
    conditions = [(COMPARISONS[c], o) for c, o in case["conditions"]]
    assert _tiles(case["length"], nb=case["batches"], conditions=conditions) == (case["visited"], case["tiles"])


def test_batches_not_a_multiple_of_the_tile_visit_at_most_their_tiles():
    visited, tiles = _tiles(100, nb=8, conditions=[(GE, 0)])
    assert tiles <= 13 * 4 and visited <= tiles


def _bounds(heaviest, largest):
    return dict(heaviest=heaviest, lightest=5e-324, largest=largest, smallest=largest, terms=3)


def _normal(heaviest, lightest, largest, smallest):
    return dict(heaviest=heaviest, lightest=lightest, largest=largest, smallest=smallest, terms=3)


def _hold(b, z, results, special):
    return oracle.bounds_hold(b["heaviest"], b["lightest"], b["largest"], b["smallest"], b["terms"], z, results,
                              special)


@pytest.mark.parametrize("case", FACTS["bounds_cases"], ids=lambda c: c["source"].rsplit(":", 1)[1])
def test_bounds_cases(case):
    assert len(FACTS["bounds_cases"]) == 15
    z = _f64(case["z"]) if case["z"] is not None else None
    got = oracle.bounds_hold(_f64(case["heaviest"]), _f64(case["lightest"]), _f64(case["largest"]),
                             _f64(case["smallest"]), case["terms"], z, [_f64(r) for r in case["results"]],
                             case["special"])
    assert got == case["holds"]


def test_signed_zeros_are_one_key_only_when_the_host_says_so():
    col = pa.array([0.0, -0.0, float("nan")])

    def same(float_keys):
        enc = oracle._encode_column(oracle.host_keys([col], float_keys)[0])
        return enc[0] == enc[1]

    assert same(oracle.SIGNED_ZEROS_EQUAL)
    assert not same(oracle.BITWISE)


def test_keys_with_long_shared_prefixes_sort_as_their_bytes():
    lp = FACTS["long_prefix"]
    prefix = lp["char"] * lp["prefix_bytes"]
    n = lp["keys"]
    strings = [f"{prefix}{i:0{lp['digits']}}" for i in reversed(range(n))]
    r = oracle.ranks_of_bytes(oracle._encode_column(pa.array(strings)))
    order = sorted(range(n), key=lambda i: strings[i])
    assert [strings[r.first[k]] for k in range(len(r.first))] == [strings[i] for i in order]
    assert np.array_equal(r.rank, np.argsort(np.argsort(strings, kind="stable"), kind="stable").astype(np.uint32))


@pytest.mark.parametrize("bits", [32, 64, 128, 256])
def test_decimal_keys_sort_as_their_values(bits):
    # Arrow's row format for decimals: big-endian, sign bit flipped.
    t = {32: pa.decimal32(9, 2), 64: pa.decimal64(18, 0), 128: pa.decimal128(38, 4), 256: pa.decimal256(76, 1)}[bits]
    top = 10 ** t.precision - 1
    vals = [0, -1, 1, top, -top, 255, -256, 256, 1 << 20, -(1 << 20), top // 3, -top // 7, None, 5, 0]
    data = b"".join((0 if v is None else v).to_bytes(t.byte_width, "little", signed=True) for v in vals)
    valid = pa.array([v is not None for v in vals]).buffers()[1]
    col = pa.Array.from_buffers(t, len(vals), [valid, pa.py_buffer(data)], null_count=1)
    r = oracle.ranks_of_bytes(oracle._encode_column(col))
    distinct = [None] + sorted({v for v in vals if v is not None})
    assert [vals[f] for f in r.first] == distinct
    assert [distinct[k] for k in r.rank] == vals


def test_dense_product_within_the_rounding_bound_and_repeatable():
    rng = oracle.Rng.seeded(11, 0)
    ni, nj, nk = 24, 300, 17
    a_vals = rng.units(ni * nj) * 2 - 1
    b_vals = rng.units(nj * nk) * 2 - 1
    sa, a = complete(["i", "j"], [ni, nj], a_vals, rng)
    sb, b = complete(["j", "k"], [nj, nk], b_vals, rng)
    f = matmul_fold()
    s = oracle.schema(f, [sa, sb])
    got = rows_of(oracle.dense_fold(f, a, b, None, s, oracle.Options(threads=1)))
    A, Bm = a_vals.reshape(ni, nj), b_vals.reshape(nj, nk)
    exact = np.array([[math.fsum(A[i] * Bm[:, k]) for k in range(nk)] for i in range(ni)]).reshape(-1)
    mag = (np.abs(A) @ np.abs(Bm)).reshape(-1)
    g = got.column(2).to_numpy()
    assert np.all(np.abs(g - exact) <= 2 * (nj - 1) * 2.0 ** -53 * mag)
    # Other batches, another order, another number of threads: the same bits.
    sa2, a2 = complete(["i", "j"], [ni, nj], a_vals, oracle.Rng.seeded(12, 0), batches=7)
    again = rows_of(oracle.dense_fold(f, a2, b, None, s, oracle.Options(threads=5)))
    assert np.array_equal(again.column(2).to_numpy().view(np.uint64), g.view(np.uint64))


@pytest.mark.parametrize("threads", [1, 3])
def test_fused_results_do_not_depend_on_threads_or_batches(threads):
    def run(seed, threads):
        case = P.attention(200, d=5, nb=2, conditions=[(GE, 0)], q_value=lambda n: oracle.Rng.seeded(1, 1).units(n),
                           v_value=lambda n: oracle.Rng.seeded(2, 1).units(n) * 2 - 1, seed=seed)
        return rows_of(P.run_oracle(case, threads=threads).batches)

    a, b = run(1, threads), run(2, 4)
    assert a.equals(b)


def test_gaussian_smoother_against_numpy():
    # The Gaussian smoother through the oracle's pipeline (against which the
    # GPU's smoother is tested): out(b, x) = sum_y w v / sum_y w with FP64 weights
    # w = exp(-power(x - y, 2) / h), computed independently with numpy.
    from einfold_b200 import cases as C

    pipe = C.smoother_pipeline(0.01)
    rng = np.random.default_rng(5)
    g, n, ny = 3, 257, 70
    x, y, v = rng.random(g * n), rng.random(g * ny), rng.standard_normal(g * ny)

    def batch(cols, names):
        return [pa.record_batch([pa.array(c) for c in cols], names=names)]

    b, t = np.repeat(np.arange(g), n), np.tile(np.arange(n), g)
    bk, tk = np.repeat(np.arange(g), ny), np.tile(np.arange(ny), g)
    qa = batch([b, t, np.zeros_like(t), x], ["b", "t", "d", "x"])
    ka = batch([bk, tk, np.zeros_like(tk), y], ["b", "t", "d", "x"])
    va = batch([bk, tk, v], ["b", "t", "x"])
    schema = oracle.pipeline_schema(pipe, [qa[0].schema, ka[0].schema, va[0].schema])
    got = oracle.pipeline(pipe, qa, ka, va, schema, oracle.Options(threads=2))
    table = rows_of(got.batches)
    assert table.num_rows == g * n
    assert np.array_equal(table.column(0).to_numpy(), b) and np.array_equal(table.column(1).to_numpy(), t)
    X, Y, V = x.reshape(g, n), y.reshape(g, ny), v.reshape(g, ny)
    w = np.exp(-(X[:, :, None] - Y[:, None, :]) ** 2 / 0.01)
    want = (np.einsum("gnk,gk->gn", w, V) / w.sum(-1)).reshape(-1)
    vals = table.column(2).to_numpy()
    assert np.abs(vals - want).max() <= 1e-13 * np.abs(want).max()
    # Tiles of 64 over the flattened positions (fused.rs:386-397): an X tile
    # pairs with the J tiles of the groups its rows belong to; every pair
    # here is allowed, so all are visited.
    tiles = 0
    for x0 in range(0, g * n, 64):
        x1 = min(x0 + 64, g * n)
        start, end = x0 // n * ny, (x1 - 1) // n * ny + ny
        tiles += -(-end // 64) - start // 64
    assert (got.tiles_visited, got.tiles) == (tiles, tiles)


def _sql(e, a, b):
    """SELECT <e> FROM a CROSS JOIN b, column by column, as SQL computes it:
    NULL wherever an operand is NULL, IEEE arithmetic on DOUBLE (division by
    zero gives ±inf or NaN), exp and ln with SQL's special values (exp's
    overflow +inf, ln of a negative NaN, of zero -inf), power as libm's pow.
    a and b: (values,
    nulls) arrays of [rows][2] for the columns x and y."""
    (av, an), (bv, bn) = a, b
    na, nb = av.shape[0], bv.shape[0]
    if e.kind == "column":
        src_v, src_n = (av, an) if e.operand == 0 else (bv, bn)
        v, n = src_v[:, e.col - 1], src_n[:, e.col - 1]
        shape = (na, 1) if e.operand == 0 else (1, nb)
        return np.broadcast_to(v.reshape(shape), (na, nb)), np.broadcast_to(n.reshape(shape), (na, nb))
    if e.kind == "literal":
        return np.full((na, nb), e.value), np.zeros((na, nb), dtype=bool)
    if e.kind == "unary":
        x, xn = _sql(e.args[0], a, b)
        with np.errstate(all="ignore"):
            if e.op is ir.Unary.NEGATE:
                v = -x
            elif e.op is ir.Unary.ABS:
                v = np.abs(x)
            elif e.op is ir.Unary.EXP:
                def exp(t):
                    try:
                        return math.exp(t)
                    except OverflowError:
                        return math.inf
                v = np.vectorize(exp, otypes=[float])(x) if x.size else x
            else:
                def ln(t):
                    if math.isnan(t) or t < 0:
                        return math.nan
                    if t == 0:
                        return -math.inf
                    return math.inf if math.isinf(t) else math.log(t)
                v = np.vectorize(ln, otypes=[float])(x) if x.size else x
        return v, xn
    x, xn = _sql(e.args[0], a, b)
    y, yn = _sql(e.args[1], a, b)
    with np.errstate(all="ignore"):
        op = e.op
        if op is ir.Binary.ADD:
            v = x + y
        elif op is ir.Binary.SUBTRACT:
            v = x - y
        elif op is ir.Binary.MULTIPLY:
            v = x * y
        elif op is ir.Binary.DIVIDE:
            v = np.divide(x, y)
        else:
            # libm's pow, as DataFusion's power (numpy's vectorised pow may
            # round otherwise): a domain error is NaN, an overflow ±inf.
            def power(p, q):
                try:
                    return math.pow(p, q)
                except ValueError:
                    return math.nan
                except OverflowError:
                    odd = q == math.floor(q) and math.fmod(q, 2.0) != 0.0
                    return -math.inf if p < 0 and odd else math.inf
            v = np.vectorize(power, otypes=[float])(x, y) if x.size else x
    return v, xn | yn


def test_evaluate_is_sqls_on_the_reference_expression_cases():
    # The reference holds Expression::evaluate to DataFusion's SQL bit for
    # bit on these cases (expression_vs_sql.rs); ir.Expression.evaluate,
    # which the device interpreter is held to, is held here to the SQL
    # evaluated column by column above.
    from tests import expression_cases as X

    def table(rows):
        v = np.zeros((len(rows), 2))
        n = np.zeros((len(rows), 2), dtype=bool)
        for i, r in enumerate(rows):
            for c in range(2):
                if r[c] is None:
                    n[i, c] = True
                else:
                    v[i, c] = r[c]
        return v, n

    pairs = 0
    for seed, rows_a, rows_b, e in X.cases():
        if not rows_a or not rows_b:
            continue
        got_v, got_n = _sql(e, table(rows_a), table(rows_b))
        for i, ra in enumerate(rows_a):
            for j, rb in enumerate(rows_b):
                rows = [ra, rb]
                want = e.evaluate(lambda o, c: rows[o][c - 1])
                pairs += 1
                assert bool(got_n[i, j]) == (want is None), (seed, i, j)
                if want is None:
                    continue
                g = float(got_v[i, j])
                same = (math.isnan(g) and math.isnan(want)) or \
                    np.float64(g).view(np.uint64) == np.float64(want).view(np.uint64)
                assert same, (seed, i, j, g, want, repr(e))
    assert pairs > 3000


def test_the_restated_property_tests_draw_the_reference_cases():
    # Each restated property test starts from the reference's seed and runs
    # its number of cases.
    from tests import expression_cases, test_dense_metamorphic_gpu, test_kernels_vs_sql_gpu, test_pipeline_vs_sql_gpu

    ours = {"kernels_vs_sql": test_kernels_vs_sql_gpu, "pipeline_vs_sql": test_pipeline_vs_sql_gpu,
            "expression_vs_sql": expression_cases, "dense_metamorphic": test_dense_metamorphic_gpu}
    for name, facts in FACTS["property_tests"].items():
        assert (ours[name].SEED, ours[name].CASES) == (facts["seed"], facts["cases"]), name
