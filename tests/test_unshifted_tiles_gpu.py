"""The unshifted tile kernel (exp weights without a shift, up to eight value
columns: a thread keeps its row's statistics and sums over all its tiles)
against the general tile kernel (EINFOLD_TILES_GENERAL=1, per-tile
half-warp reductions) and the oracle (fused.rs restated): the same rows,
tile counts and declines, values within 1e-12·max|v| of the oracle and
within 1e-14 of the general kernel's (the sums add the same terms in
another order)."""
import numpy as np
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests import pipelines as P
from tests.tables import rows_of

pytestmark = pytest.mark.gpu

GE, LT = ir.Comparison.GREATER_OR_EQUAL, ir.Comparison.LESS


def _run(case, general, monkeypatch):
    if general:
        monkeypatch.setenv("EINFOLD_TILES_GENERAL", "1")
    else:
        monkeypatch.delenv("EINFOLD_TILES_GENERAL", raising=False)
    got = K.pipeline(case.pipeline, [K.Relation(*case.q), K.Relation(*case.k), K.Relation(*case.v)])
    monkeypatch.delenv("EINFOLD_TILES_GENERAL", raising=False)
    return got


def _values(got):
    t = rows_of(got.batches)
    return t, t.column(t.num_columns - 1).to_numpy(zero_copy_only=False)


def _check(case, monkeypatch):
    want = P.run_oracle(case)
    fast = _run(case, False, monkeypatch)
    slow = _run(case, True, monkeypatch)
    if want is None:
        assert fast is None and slow is None
        return
    assert fast is not None and slow is not None
    assert (fast.tiles_visited, fast.tiles) == (slow.tiles_visited, slow.tiles) == (want.tiles_visited, want.tiles)
    ft, fv = _values(fast)
    st, sv = _values(slow)
    wt, wv = _values(want)
    assert ft.num_rows == st.num_rows == wt.num_rows
    for c in range(ft.num_columns - 1):
        assert ft.column(c).equals(wt.column(c)) and st.column(c).equals(wt.column(c))
    assert np.array_equal(np.isnan(fv), np.isnan(wv)) and np.array_equal(np.isnan(sv), np.isnan(wv))
    inf = np.isinf(wv)
    assert np.array_equal(fv[inf], wv[inf])
    fin = np.isfinite(wv)
    scale = max(case.v_scale, 1e-300)
    if case.pipeline.normalizer() == ir.Normalizer.NONE:
        scale = max(np.abs(wv[fin]).max(initial=0.0), 1e-300)
    assert np.all(np.abs(fv[fin] - wv[fin]) <= 1e-12 * scale)
    assert np.all(np.abs(fv[fin] - sv[fin]) <= 1e-14 * scale)


@pytest.mark.parametrize("scores", ["product", "gaussian", "interpreted"])
@pytest.mark.parametrize("normalizer", [ir.Normalizer.KEPT_GROUPS, ir.Normalizer.JOINED_ROWS, ir.Normalizer.NONE])
def test_unshifted_weights_give_the_general_kernels_results(scores, normalizer, monkeypatch):
    expr = {"product": None, "gaussian": P.gaussian_scores(),
            "interpreted": ir.Expression.column(0, -1).binary(ir.Binary.MULTIPLY, ir.Expression.column(1, -1))
            .unary(ir.Unary.NEGATE).unary(ir.Unary.ABS)}[scores]
    d = 1 if scores == "gaussian" else 5
    scale = ir.Scale.over(0.05) if scores == "gaussian" else ir.Scale.times(0.5)
    case = P.attention(150, d=d, lk=110, nb=2, c=3, scores=expr, conditions=[(GE, -30), (LT, 60)],
                       weight=ir.Weight.exp(scale, ir.Shift.NONE), normalizer=normalizer,
                       q_value=lambda n: oracle.Rng.seeded(31, 2).units(n),
                       k_value=lambda n: oracle.Rng.seeded(32, 2).units(n),
                       v_value=lambda n: oracle.Rng.seeded(33, 2).units(n) * 2 - 1)
    _check(case, monkeypatch)


def test_one_value_column_and_no_mask(monkeypatch):
    case = P.attention(200, d=1, lk=70, nb=3, scores=P.gaussian_scores(),
                       weight=ir.Weight.exp(ir.Scale.over(0.01), ir.Shift.NONE),
                       q_value=lambda n: oracle.Rng.seeded(34, 2).units(n),
                       k_value=lambda n: oracle.Rng.seeded(35, 2).units(n),
                       v_value=lambda n: oracle.Rng.seeded(36, 2).units(n) * 2 - 1)
    _check(case, monkeypatch)


def test_special_values_and_overflow_decline_alike(monkeypatch):
    rng = oracle.Rng.seeded(37, 2)

    def with_specials(n, scale):
        x = (rng.units(n) * 2 - 1) * scale
        for i in range(0, n, 89):
            x[i] = [np.nan, np.inf, -np.inf, 1e300, -1e300][(i // 89) % 5]
        return x

    for normalizer in (ir.Normalizer.KEPT_GROUPS, ir.Normalizer.NONE):
        for target in ("q", "v"):
            case = P.attention(
                120, d=4, nb=2, c=2, conditions=[(GE, 0)], normalizer=normalizer,
                weight=ir.Weight.exp(ir.Scale.one(), ir.Shift.NONE),
                q_value=(lambda n: with_specials(n, 2)) if target == "q" else (lambda n: rng.units(n)),
                v_value=(lambda n: with_specials(n, 1)) if target == "v" else (lambda n: rng.units(n) * 2 - 1))
            _check(case, monkeypatch)
    # Each weight exp(709) finite, their sum not: both kernels decline.
    case = P.attention(64, d=1, weight=ir.Weight.exp(ir.Scale.one(), ir.Shift.NONE),
                       q_value=lambda n: np.full(n, np.sqrt(709.0)), k_value=lambda n: np.full(n, np.sqrt(709.0)))
    _check(case, monkeypatch)
