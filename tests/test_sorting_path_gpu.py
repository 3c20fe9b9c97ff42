"""The sorting path at its configuration: a sparse contraction with
non-positional keys (i and k 16-hex-digit strings from 50,000 distinct, j a
63-bit hash from a pool of 200,000 with Zipf(1.1) frequencies, v normal), and
its regridding variant (a weighted by w(src, dst, wt)), on the GPU against
the oracle's restatement of discriminate::fold (discriminate.rs:369-650):

- at 1/40 of the tables' size, the whole result: keys, group order and
  values bit for bit;
- at full size (2M + 2M rows), the ranks of j over a‖b, of i and of k bit for
  bit, and the groups of sampled x-blocks (the result's rows of a few values
  of i, which depend only on a's rows with those i and on b:
  discriminate.rs:548-584 sums each block of x apart) bit for bit;
- the regridding variant at 1/80 of its size, the whole result bit for bit.
"""
import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

from einfold_b200 import ir, kernels as K, synthetic as S
from oracle import oracle
from tests.tables import assert_same_rows, matmul_fold, rows_of

pytestmark = pytest.mark.gpu


def _oracle_fold(f, a, b):
    return oracle.fold(f, a.schema, [a], b.schema, [b], None, oracle.schema(f, [a.schema, b.schema]))


def test_the_sparse_tables_at_one_fortieth_give_the_oracles_rows():
    a, b = S.sorting_tables(50_000)
    f = matmul_fold()
    got = K.fold(f, K.Relation(a.schema, [a]), K.Relation(b.schema, [b]))
    want = _oracle_fold(f, a, b)
    assert got.algorithm == K.Algorithm.DISCRIMINATE and want.algorithm == "discriminate"
    g, w = rows_of(got.batches), rows_of(want.batches)
    assert g.num_rows > 50_000_000
    assert_same_rows(g, w, exact=True)


def _unique_ranks(values):
    """Ranks and first rows by numpy, independently of both implementations."""
    u, first, inv = np.unique(values, return_index=True, return_inverse=True)
    return inv.astype(np.uint32), first.astype(np.uint32)


def test_full_size_ranks_of_j_i_and_k():
    a, b = S.sorting_tables()
    j = pa.concat_arrays([a.column(1), b.column(0)])
    rel = lambda col, name: K.Relation(pa.schema([(name, col.type)]), [pa.record_batch([col], names=[name])])
    got = K.rank_columns(rel(j, "j"), [0])
    want = oracle.rank_columns([j], len(j))
    assert np.array_equal(got.rank, want.rank) and np.array_equal(got.first, want.first)
    r, f = _unique_ranks(j.to_numpy())
    assert np.array_equal(got.rank, r) and np.array_equal(got.first, f)
    for col, name in ((a.column(0), "i"), (b.column(1), "k")):
        got = K.rank_columns(rel(col, name), [0])
        # 16-byte strings order as their bytes: numpy's fixed-width byte strings.
        r, f = _unique_ranks(np.asarray(col.to_numpy(zero_copy_only=False), dtype="S16"))
        assert np.array_equal(got.rank, r) and np.array_equal(got.first, f)
        assert len(got.first) == len(np.unique(np.asarray(col.to_numpy(zero_copy_only=False), dtype="S16")))


def test_full_size_sampled_x_blocks():
    a, b = S.sorting_tables()
    names = pc.unique(a.column(0))
    rng = oracle.Rng.seeded(41, 0)
    sample = pa.array(sorted({names[rng.below(len(names))].as_py() for _ in range(12)}))
    a_s = a.filter(pc.is_in(a.column(0), value_set=sample))
    # b whole on the GPU; for the oracle, only b's rows that join a sampled
    # row (the others add no term to these groups).
    b_s = b.filter(pc.is_in(b.column(0), value_set=pc.unique(a_s.column(1))))
    f = matmul_fold()
    got = K.fold(f, K.Relation(a_s.schema, [a_s]), K.Relation(b.schema, [b]))
    want = _oracle_fold(f, a_s, b_s)
    g, w = rows_of(got.batches), rows_of(want.batches)
    assert g.num_rows > 10_000
    seen = set(pc.unique(g.column(0)).to_pylist())
    assert seen <= set(sample.to_pylist()) and len(seen) >= 10
    assert_same_rows(g, w, exact=True)


def test_the_regridding_variant_gives_the_oracles_rows():
    a, _ = S.sorting_tables(50_000)
    wt = S.regrid_table(50_000)
    w = pa.record_batch([wt.column(0), wt.column(1), wt.column(2)], names=["j", "k", "v"])
    f = matmul_fold()
    got = K.fold(f, K.Relation(a.schema, [a]), K.Relation(w.schema, [w]))
    want = _oracle_fold(f, a, w)
    assert got.algorithm == K.Algorithm.DISCRIMINATE
    g = rows_of(got.batches)
    assert g.column(1).type == pa.int64() and g.num_rows > 1_000_000
    assert_same_rows(g, rows_of(want.batches), exact=True)
