"""The fused pipeline on the GPU against the oracle (fused.rs restated): the
same rows, the same tile counts, the same declines, and values within
1e-12·max|v| — the reference's own property bound is 1e-9·max|v|
(pipeline_vs_sql.rs:36-39); the scores' and sums' order of rounding is the
kernel's, as the reference's GEMM's is matrixmultiply's."""
import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests import pipelines as P
from tests.tables import reference_facts, rows_of

pytestmark = pytest.mark.gpu

GE, GT, LE, LT = (ir.Comparison.GREATER_OR_EQUAL, ir.Comparison.GREATER, ir.Comparison.LESS_OR_EQUAL,
                  ir.Comparison.LESS)
TOL = 1e-12


def _gpu(case: P.Case, options=None):
    return K.pipeline(case.pipeline, [K.Relation(*case.q), K.Relation(*case.k), K.Relation(*case.v)],
                      options=options)


def _same(case: P.Case, tol: float = TOL, options=None):
    want = P.run_oracle(case)
    got = _gpu(case, options)
    if want is None:
        assert got is None
        return None
    assert got is not None, "the GPU declined what the oracle computes"
    assert (got.tiles_visited, got.tiles) == (want.tiles_visited, want.tiles)
    g, w = rows_of(got.batches), rows_of(want.batches)
    assert g.num_rows == w.num_rows and g.schema == w.schema
    for c in range(g.num_columns - 1):
        assert g.column(c).equals(w.column(c)), f"key column {c} differs"
    gv = g.column(g.num_columns - 1).to_numpy(zero_copy_only=False)
    wv = w.column(w.num_columns - 1).to_numpy(zero_copy_only=False)
    assert np.array_equal(np.isnan(gv), np.isnan(wv)), "NaNs differ"
    inf = np.isinf(wv)
    assert np.array_equal(gv[inf], wv[inf]), "infinities differ"
    fin = np.isfinite(wv)
    err = np.abs(gv[fin] - wv[fin])
    if case.pipeline.normalizer() == ir.Normalizer.NONE:
        # A sum that nothing normalizes: each group's scale is its Σ|w·v|,
        # the same pipeline over |v| (every weight here is nonnegative).
        scale = _magnitudes(case)[fin]
    else:
        scale = max(case.v_scale, 1e-300)
    assert np.all(err <= tol * scale), f"worst {np.max(err / np.maximum(scale, 1e-300)):.3e} of the scale"
    return got


def _magnitudes(case: P.Case) -> np.ndarray:
    sv, bv = case.v

    def absolute(b):
        cols = list(b.columns)
        cols[-1] = pa.array(np.abs(cols[-1].to_numpy(zero_copy_only=False)), pa.float64())
        return pa.RecordBatch.from_arrays(cols, schema=sv)

    m = P.run_oracle(P.Case(case.pipeline, case.q, case.k, (sv, [absolute(b) for b in bv]), case.v_scale))
    t = rows_of(m.batches)
    return np.abs(t.column(t.num_columns - 1).to_numpy(zero_copy_only=False))


@pytest.mark.parametrize("case", reference_facts()["tile_counts"], ids=lambda c: c["test"])
def test_masks_and_batches_visit_the_reference_tile_counts(case):
    comparisons = {"ge": GE, "gt": GT, "le": LE, "lt": LT}
    conditions = [(comparisons[c], o) for c, o in case["conditions"]]
    got = _same(P.attention(case["length"], nb=case["batches"], conditions=conditions))
    assert (got.tiles_visited, got.tiles) == (case["visited"], case["tiles"])


def test_batches_not_a_multiple_of_the_tile():
    _same(P.attention(100, nb=8, conditions=[(GE, 0)]))


@pytest.mark.parametrize("mirrored", [False, True])
@pytest.mark.parametrize("conditions", [[], [(GE, 0)], [(GT, -3)], [(LE, 5), (GT, -40)], [(LT, 0)],
                                        [(GE, 0), (LT, 1)], [(GE, 200)]])
def test_attention_with_spread_scores_and_masks(conditions, mirrored):
    case = P.attention(150, d=16, nb=3, c=5, conditions=conditions, mirrored=mirrored,
                       q_value=lambda n: (oracle.Rng.seeded(1, 2).units(n) * 2 - 1) * 3,
                       k_value=lambda n: (oracle.Rng.seeded(2, 2).units(n) * 2 - 1) * 3,
                       v_value=lambda n: oracle.Rng.seeded(3, 2).units(n) * 2 - 1)
    _same(case)


@pytest.mark.parametrize("scale", [ir.Scale.one(), ir.Scale.times(0.125), ir.Scale.over(8.0)])
@pytest.mark.parametrize("shift", [ir.Shift.KEPT_MAXIMUM, ir.Shift.NONE])
@pytest.mark.parametrize("normalizer", [ir.Normalizer.KEPT_GROUPS, ir.Normalizer.JOINED_ROWS, ir.Normalizer.NONE])
def test_softmax_scales_shifts_and_normalizers(scale, shift, normalizer):
    case = P.attention(130, d=40, nb=2, c=3, conditions=[(GE, 0)], weight=ir.Weight.exp(scale, shift),
                       normalizer=normalizer,
                       q_value=lambda n: oracle.Rng.seeded(4, 2).units(n) * 2 - 1,
                       k_value=lambda n: oracle.Rng.seeded(5, 2).units(n) * 2 - 1,
                       v_value=lambda n: oracle.Rng.seeded(6, 2).units(n) * 2 - 1)
    _same(case)


@pytest.mark.parametrize("weight", ["sigmoid", "cauchy"])
@pytest.mark.parametrize("normalizer", [ir.Normalizer.KEPT_GROUPS, ir.Normalizer.NONE])
def test_expression_weights(weight, normalizer):
    w = P.sigmoid_weight() if weight == "sigmoid" else P.cauchy_weight()
    case = P.attention(140, d=6, nb=2, conditions=[(GE, 0), (LT, 70)], weight=ir.Weight.of_expression(w),
                       normalizer=normalizer,
                       q_value=lambda n: oracle.Rng.seeded(7, 2).units(n) * 2 - 1,
                       k_value=lambda n: oracle.Rng.seeded(8, 2).units(n) * 2 - 1,
                       v_value=lambda n: oracle.Rng.seeded(9, 2).units(n) * 2 - 1)
    _same(case)


def test_gaussian_smoother_scores_are_a_row_expression():
    # exp(-power(x - y, 2) / h) with h = 0.01: scores -power(q.x - k.x, 2)
    # over one feature, weights a softmax of the scores over h.
    case = P.attention(300, d=1, lk=90, nb=2, scores=P.gaussian_scores(),
                       weight=ir.Weight.exp(ir.Scale.over(0.01), ir.Shift.KEPT_MAXIMUM),
                       q_value=lambda n: oracle.Rng.seeded(10, 2).units(n),
                       k_value=lambda n: oracle.Rng.seeded(11, 2).units(n),
                       v_value=lambda n: oracle.Rng.seeded(12, 2).units(n) * 2 - 1)
    _same(case)


def test_many_values_and_features_span_chunks():
    # 130 value columns (three chunks of 64) and 70 features (three of 32).
    case = P.attention(70, d=70, c=130, conditions=[(GE, 0)],
                       q_value=lambda n: (oracle.Rng.seeded(13, 2).units(n) * 2 - 1) * 0.3,
                       k_value=lambda n: (oracle.Rng.seeded(14, 2).units(n) * 2 - 1) * 0.3,
                       v_value=lambda n: oracle.Rng.seeded(15, 2).units(n) * 2 - 1)
    _same(case)


def test_special_values_give_the_oracles_result_or_decline_alike():
    rng = oracle.Rng.seeded(16, 2)

    def with_specials(n, scale):
        x = (rng.units(n) * 2 - 1) * scale
        for i in range(0, n, 97):
            x[i] = [np.nan, np.inf, -np.inf, 1e300, -1e300][(i // 97) % 5]
        return x

    for normalizer in (ir.Normalizer.KEPT_GROUPS, ir.Normalizer.NONE):
        for target in ("q", "v"):
            case = P.attention(
                120, d=4, nb=2, c=2, conditions=[(GE, 0)], normalizer=normalizer,
                q_value=(lambda n: with_specials(n, 2)) if target == "q" else (lambda n: rng.units(n)),
                v_value=(lambda n: with_specials(n, 1)) if target == "v" else (lambda n: rng.units(n) * 2 - 1))
            _same(case)


def test_scores_that_overflow_exp_decline_alike():
    # Unshifted weights exp(s) with s = 709: each weight is finite, their
    # sum is not.
    case = P.attention(64, d=1, weight=ir.Weight.exp(ir.Scale.one(), ir.Shift.NONE),
                       q_value=lambda n: np.full(n, np.sqrt(709.0)), k_value=lambda n: np.full(n, np.sqrt(709.0)))
    assert P.run_oracle(case) is None
    assert _gpu(case) is None


def test_all_minus_infinity_rows_are_nan():
    q = lambda n: np.where(np.arange(n) < 16, -np.inf, 1.0)  # the first rows' scores are -inf
    for normalizer in (ir.Normalizer.KEPT_GROUPS, ir.Normalizer.NONE):
        case = P.attention(40, d=2, normalizer=normalizer, q_value=q, k_value=lambda n: np.full(n, 0.5))
        _same(case)


def _decline(case: P.Case):
    assert P.run_oracle(case) is None
    assert _gpu(case) is None


def test_declines_a_repeated_or_missing_row_or_a_null_factor():
    case = P.attention(50, d=3)
    sq, bq = case.q
    _decline(P.Case(case.pipeline, (sq, bq + [bq[0].slice(0, 1)]), case.k, case.v, 1.0))  # repeated
    _decline(P.Case(case.pipeline, (sq, [b.slice(1) if i == 0 else b for i, b in enumerate(bq)]), case.k, case.v,
                    1.0))  # missing
    sv, bv = case.v
    nulled = []
    for i, b in enumerate(bv):
        cols = list(b.columns)
        if i == 0 and b.num_rows:
            vals = cols[-1].to_pylist()
            vals[0] = None
            cols[-1] = pa.array(vals, pa.float64())
        nulled.append(pa.RecordBatch.from_arrays(cols, schema=sv))
    _decline(P.Case(case.pipeline, case.q, case.k, (sv, nulled), 1.0))


def test_declines_a_pipeline_that_sums_its_own_dimension_away():
    case = P.attention(8, d=2, c=3)
    p = case.pipeline
    p2 = ir.Pipeline(p.producer(), p.weight(), p.dimensions(), p.values(), [o for o in p.outputs() if o < 3],
                     p.normalizer())
    _decline(P.Case(p2, case.q, case.k, case.v, 1.0))


def test_empty_relations():
    case = P.attention(0, d=2)
    got, want = _gpu(case), P.run_oracle(case)
    assert (got is None) == (want is None)
    if got is not None:
        assert rows_of(got.batches).num_rows == rows_of(want.batches).num_rows == 0


def test_results_left_in_hbm_match_the_host_result():
    # result_on_device: the same rows as the host result, as DeviceBatch
    # columns (the Gaussian smoother's pipeline, two batches of positions).
    import torch

    case = P.attention(300, d=1, lk=90, nb=2, scores=P.gaussian_scores(),
                       weight=ir.Weight.exp(ir.Scale.over(0.01), ir.Shift.NONE),
                       q_value=lambda n: oracle.Rng.seeded(10, 3).units(n),
                       k_value=lambda n: oracle.Rng.seeded(11, 3).units(n),
                       v_value=lambda n: oracle.Rng.seeded(12, 3).units(n) * 2 - 1)
    host = rows_of(_gpu(case).batches)
    got = _gpu(case, K.Options(result_on_device=True))
    try:
        assert len(got.batches) == 1 and isinstance(got.batches[0], K.DeviceBatch)
        dev = got.batches[0]
        assert dev.rows == host.num_rows
        for c in range(host.num_columns):
            assert np.array_equal(dev.column(c).cpu().numpy(), host.column(c).to_numpy()), f"column {c}"
        assert isinstance(dev.column(0), torch.Tensor)
    finally:
        for b in got.batches:
            b.release()


def _bits(case: P.Case):
    got = rows_of(_gpu(case).batches)
    return got.column(got.num_columns - 1).to_numpy(zero_copy_only=False)


@pytest.mark.parametrize("shape", ["gaussian", "sigmoid", "cauchy"])
def test_named_shapes_give_the_interpreters_bits(shape):
    # The kernel computes -power(a - b, 2) scores and the sigmoid and Cauchy
    # weights without its expression interpreter; the same expressions
    # written in another order of the same operations take the interpreter.
    s = ir.Expression.column(0, 0)
    one = ir.Expression.literal(1.0)
    a, b = ir.Expression.column(0, -1), ir.Expression.column(1, -1)
    diff = a.binary(ir.Binary.SUBTRACT, b)
    kw = dict(q_value=lambda n: oracle.Rng.seeded(17, 2).units(n) * 2 - 1,
              k_value=lambda n: oracle.Rng.seeded(18, 2).units(n) * 2 - 1,
              v_value=lambda n: oracle.Rng.seeded(19, 2).units(n) * 2 - 1)
    if shape == "gaussian":
        fast = diff.binary(ir.Binary.POWER, ir.Expression.literal(2.0)).unary(ir.Unary.NEGATE)
        slow = diff.unary(ir.Unary.NEGATE).binary(ir.Binary.MULTIPLY, diff)  # (-d)·d = -(d·d)
        cases = [P.attention(200, d=3, lk=130, nb=2, scores=e, conditions=[(GE, -40)],
                             weight=ir.Weight.exp(ir.Scale.over(0.05), ir.Shift.KEPT_MAXIMUM), **kw)
                 for e in (fast, slow)]
    else:
        if shape == "sigmoid":
            tail = s.unary(ir.Unary.NEGATE).unary(ir.Unary.EXP)
        else:
            tail = s.binary(ir.Binary.MULTIPLY, s)
        fast = one.binary(ir.Binary.DIVIDE, one.binary(ir.Binary.ADD, tail))
        slow = one.binary(ir.Binary.DIVIDE, tail.binary(ir.Binary.ADD, one))  # the sum's operands swapped
        cases = [P.attention(150, d=5, nb=2, conditions=[(GE, 0), (LT, 90)], weight=ir.Weight.of_expression(e),
                             **kw) for e in (fast, slow)]
    got_fast, got_slow = (_bits(c) for c in cases)
    assert np.array_equal(got_fast.view(np.uint64), got_slow.view(np.uint64))
    _same(cases[0])


def test_gaussian_smoother_at_scale_against_torch_float64():
    # The Gaussian smoother at 4 groups of 65,536 x and 256 y (67 M pairs,
    # tables in HBM, result left there): every row against torch float64.
    import torch

    from einfold_b200 import cases as C

    groups, nx, ny, h = 4, 1 << 16, 256, 0.01
    q, k, v, xs, ys, vs = C.smoother_tables(groups, nx, ny, seed=3)
    got = K.pipeline(C.smoother_pipeline(h), [q, k, v], options=K.Options(result_on_device=True))
    try:
        vals = got.batches[0].column(2).view(groups, nx)
        X, Y, V = xs.view(groups, nx), ys.view(groups, ny), vs.view(groups, ny)
        w = torch.exp(-(X[:, :, None] - Y[:, None, :]) ** 2 / h)
        want = torch.einsum("gnk,gk->gn", w, V) / w.sum(-1)
        assert got.batches[0].rows == groups * nx
        assert ((vals - want).abs().max() / want.abs().max()).item() <= 1e-13
    finally:
        for b in got.batches:
            b.release()
