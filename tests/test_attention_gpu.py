"""The split form of attention-shaped pipelines (int8 digit products on the
tensor cores, FP64 softmax) against the FP64 tile kernel and the oracle:
the same rows and tile counts, values within 1e-12·max|v|, and the tensor
path verifiably taken."""
import dataclasses

import numpy as np
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests import pipelines as P
from tests.tables import rows_of

pytestmark = pytest.mark.gpu

GE, LT = ir.Comparison.GREATER_OR_EQUAL, ir.Comparison.LESS


def _normal(seed, sd):
    def draw(n):
        rng = oracle.Rng.seeded(seed, 3)
        u1, u2 = rng.units(n), rng.units(n)
        return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2 * np.pi * u2) * sd
    return draw


def _run(case, precision, slices=0):
    opts = K.Options(precision=precision, slices=slices)
    got = K.pipeline(case.pipeline, [K.Relation(*case.q), K.Relation(*case.k), K.Relation(*case.v)], options=opts)
    return got, dataclasses.replace(K.last_call)


def _values(piped):
    t = rows_of(piped.batches)
    return t, t.column(t.num_columns - 1).to_numpy(zero_copy_only=False)


CASES = {
    # batch·head groups, query and key length, features, value columns, conditions
    "causal_d64": dict(nb=4, l=512, d=64, conditions=[(GE, 0)]),
    "ragged_window": dict(nb=3, l=300, d=64, conditions=[(GE, 0), (LT, 96)]),
    "causal_d128": dict(nb=2, l=200, d=128, conditions=[(GE, 0)]),
    "two_value_chunks": dict(nb=2, l=130, d=64, c=100, conditions=[(GE, 0)]),
    "cross_lengths": dict(nb=1, l=256, lk=384, d=32),
    "single_rows": dict(nb=5, l=1, d=8),
}


@pytest.mark.parametrize("name", list(CASES))
def test_split_attention_matches_the_fp64_tiles(name):
    kw = CASES[name]
    slices = 6
    case = P.attention(**kw, q_value=_normal(1, 0.125 * 4), k_value=_normal(2, 0.125 * 4),
                       v_value=_normal(3, 0.125))
    split, info = _run(case, K.Precision.SPLIT, slices)
    assert info.product_ops > 0, "the tensor-core path didn't run"
    fp64, info64 = _run(case, K.Precision.FP64)
    assert info64.product_ops == 0
    assert (split.tiles_visited, split.tiles) == (fp64.tiles_visited, fp64.tiles)
    ts, vs = _values(split)
    tf, vf = _values(fp64)
    assert ts.num_rows == tf.num_rows
    for c in range(ts.num_columns - 1):
        assert ts.column(c).equals(tf.column(c))
    scale = case.v_scale
    assert np.max(np.abs(vs - vf)) <= 1e-12 * scale, np.max(np.abs(vs - vf)) / scale
    if name in ("ragged_window", "causal_d128", "single_rows"):
        want = P.run_oracle(case)
        assert (want.tiles_visited, want.tiles) == (split.tiles_visited, split.tiles)
        _, vo = _values(want)
        assert np.max(np.abs(vs - vo)) <= 1e-12 * scale


@pytest.mark.parametrize("slices,tol", [(6, 1e-10)])
def test_peaked_softmax(slices, tol):
    # Scores spread over hundreds: most weights underflow toward 0 and the
    # average follows a few keys. A score's error is absolute, about
    # ne·2^(3-8S)·max|q|·max|k|, and exp turns it into a relative error of
    # the weights: six slices keep 1e-10 of max|v| here (the reference's own
    # bound is 1e-9).
    case = P.attention(nb=2, l=256, d=16, conditions=[(GE, 0)], q_value=_normal(4, 6.0), k_value=_normal(5, 6.0),
                       v_value=_normal(6, 1.0))
    split, info = _run(case, K.Precision.SPLIT, slices)
    assert info.product_ops > 0
    fp64, _ = _run(case, K.Precision.FP64)
    _, vs = _values(split)
    _, vf = _values(fp64)
    assert np.max(np.abs(vs - vf)) <= tol * case.v_scale


def test_other_slice_counts_take_the_fp64_tiles():
    # The split attention runs six slices: their levels and the rows' sums
    # fill TMEM.
    case = P.attention(nb=2, l=100, d=8, conditions=[(GE, 0)], q_value=_normal(8, 0.5))
    got, info = _run(case, K.Precision.SPLIT, 7)
    assert info.product_ops == 0
    want, _ = _run(case, K.Precision.FP64)
    _, vg = _values(got)
    _, vw = _values(want)
    assert np.array_equal(vg, vw)


def test_nonfinite_operands_take_the_fp64_tiles():
    q = _normal(7, 0.5)

    def with_nan(n):
        x = q(n)
        x[5] = np.nan
        return x

    case = P.attention(nb=2, l=100, d=8, conditions=[(GE, 0)], q_value=with_nan)
    got, info = _run(case, K.Precision.SPLIT)
    assert info.product_ops == 0
    want = P.run_oracle(case)
    _, vg = _values(got)
    _, vw = _values(want)
    assert np.array_equal(np.isnan(vg), np.isnan(vw))
