"""Chains of three operands on the GPU against the oracle's restatement of
chain.rs: the same rows and declines; in the FP64 form the same bits (each
of the two dense folds adds in the reference's order), in the split form
within the split product's bound."""
import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests.tables import assert_same_rows, complete, rows_of

pytestmark = pytest.mark.gpu

E = ir.EQ


def _chain(outputs=(0, 3)):
    """SUM(a.v * b.v * c.v) over a(i, j) JOIN b(j, k) JOIN c(k, l) GROUP BY outputs."""
    return ir.Fold([E, E, E, E], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2),
                                  ir.Operand([(2, 0), (3, 1)], 2)], [ir.Output(d) for d in outputs])


def _tables(ni, nj, nk, nl, seed, nulls_c=0.0, scale=1.0):
    rng = oracle.Rng.seeded(seed, 0)
    a = complete(["i", "j"], [ni, nj], (rng.units(ni * nj) * 2 - 1) * scale, rng)
    b = complete(["j", "k"], [nj, nk], (rng.units(nj * nk) * 2 - 1) * scale, rng)
    c = complete(["k", "l"], [nk, nl], (rng.units(nk * nl) * 2 - 1) * scale, rng,
                 nulls=rng.units(nk * nl) < nulls_c if nulls_c else None)
    return [a, b, c]


def _both(f, tables, precision):
    schemas = [s for s, _ in tables]
    out_schema = oracle.schema(f, schemas)
    want = oracle.fold_chain(f, tables, out_schema)
    got = K.fold_chain(f, [K.Relation(s, b) for s, b in tables], options=K.Options(precision=precision))
    return got, want


@pytest.mark.parametrize("shape", [(50, 40, 3, 60), (3, 40, 50, 60), (64, 64, 64, 64), (1, 7, 1, 5)])
def test_chains_match_the_oracle_bit_for_bit_in_fp64(shape):
    tables = _tables(*shape, seed=sum(shape))
    got, want = _both(_chain(), tables, K.Precision.FP64)
    assert want is not None and got is not None
    assert_same_rows(rows_of(got), rows_of(want), exact=True)


@pytest.mark.parametrize("outputs", [(0, 3), (0,), (3, 0), (1, 3)])
def test_chains_in_the_split_form(outputs):
    tables = _tables(60, 50, 40, 30, seed=3)
    got, want = _both(_chain(outputs), tables, K.Precision.SPLIT)
    if want is None:  # the dense fold declines a step of this chain
        assert got is None
        return
    w = rows_of(want)
    scale = np.abs(w.column(w.num_columns - 1).to_numpy(zero_copy_only=False)).max()
    # Two split products, each within ~1e-13 of its terms' scale here.
    assert_same_rows(rows_of(got), w, tol=1e-12 * max(scale, 1.0))


def test_holes_in_one_operand_swap_the_dense_folds_operands():
    tables = _tables(20, 30, 25, 15, seed=5, nulls_c=0.05)
    got, want = _both(_chain(), tables, K.Precision.FP64)
    assert want is not None and got is not None
    assert_same_rows(rows_of(got), rows_of(want), exact=True)


def test_declines_like_the_reference():
    base = _tables(10, 12, 8, 9, seed=7)
    # A factor that isn't finite.
    s, b = base[1]
    vals = np.concatenate([x.column(2).to_numpy(zero_copy_only=False) for x in b])
    vals[3] = np.inf
    col = pa.array(vals)
    bad = [(s, [pa.RecordBatch.from_arrays([pa.concat_arrays([x.column(0) for x in b]),
                                            pa.concat_arrays([x.column(1) for x in b]), col], schema=s)])]
    for tables in ([base[0], bad[0], base[2]],
                   _tables(10, 12, 8, 9, seed=8, scale=1e120)):  # Π max|f|·rows above 2^1000
        got, want = _both(_chain(), tables, K.Precision.FP64)
        assert want is None and got is None
    # A condition, or two operands only.
    with_cond = _chain().with_conditions([ir.Condition(0, ir.Comparison.LESS, 3, 0)])
    got, want = _both(with_cond, base, K.Precision.FP64)
    assert want is None and got is None
