"""Key types on the GPU path beyond integers, floats and strings: dates,
times, timestamps and durations rank, join and group as their values (the
reference ranks every type by Arrow's row format, keys.rs:16-37) and come
back with their own types; the dense algorithm, which takes integer keys
only (dense.rs:93-110), declines them; a column of a type the library can't
read is allowed where no call reads it, and a key of such a type declines to
the host plan."""

import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K

pytestmark = pytest.mark.gpu

E = ir.Dimension(ir.KeyEquality.EQUAL)


def _fold(domain=False):
    # SUM(a.v * b.v) over a(i, j) JOIN b(j, k) GROUP BY i, k.
    outs = [ir.Output(0, ir.DomainKey(0) if domain else None), ir.Output(2, ir.DomainKey(1) if domain else None)]
    return ir.Fold([E, E, E], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)], outs,
                   domain=ir.Domain((0, 1), None) if domain else None)


def _rel(cols, names):
    b = pa.record_batch(cols, names=names)
    return K.Relation(b.schema, [b.slice(0, b.num_rows // 2), b.slice(b.num_rows // 2)])


def _as_int(col):
    # A temporal column's values as integers (32-bit types through int32).
    if pa.types.is_date32(col.type) or pa.types.is_time32(col.type):
        col = col.cast(pa.int32())
    return col.cast(pa.int64()).to_pylist()


def _rows(batches):
    t = pa.Table.from_batches(batches)
    keys = list(zip(*[_as_int(t.column(c)) for c in range(t.num_columns - 1)]))
    vals = t.column(t.num_columns - 1).to_pylist()
    return sorted(zip(keys, vals), key=lambda r: r[0]), t.schema


def _inputs(seed=3):
    rng = np.random.default_rng(seed)
    n, m = 4000, 300
    i = rng.integers(-20_000, 20_000, n)  # days around the epoch
    j = rng.integers(0, 60, n)
    j2 = rng.integers(0, 60, m)
    k = rng.integers(-(1 << 40), 1 << 40, m) * 1000  # microseconds
    k[::7] = k[3]  # repeated keys
    return i, j, rng.normal(size=n), j2, k, rng.normal(size=m)


@pytest.mark.parametrize("k_type", [pa.timestamp("us", tz="UTC"), pa.duration("us"), pa.time64("us"), pa.date64()])
def test_temporal_keys_group_as_their_values(k_type):
    i, j, va, j2, k, vb = _inputs()
    if k_type == pa.time64("us"):
        k = np.abs(k) % (86_400 * 10 ** 6)
    if k_type == pa.date64():
        k = (k // 86_400_000) * 86_400_000
    a_t = _rel([pa.array(i, pa.int32()).cast(pa.date32()), pa.array(j), pa.array(va)], ["i", "j", "v"])
    b_t = _rel([pa.array(j2), pa.array(k, pa.int64()).cast(k_type), pa.array(vb)], ["j", "k", "v"])
    a_i = _rel([pa.array(i, pa.int32()), pa.array(j), pa.array(va)], ["i", "j", "v"])
    b_i = _rel([pa.array(j2), pa.array(k, pa.int64()), pa.array(vb)], ["j", "k", "v"])
    f = _fold()
    got = K.fold(f, a_t, b_t, options=K.Options(precision=K.Precision.FP64))
    want = K.fold(f, a_i, b_i, options=K.Options(precision=K.Precision.FP64))
    assert got.algorithm == K.Algorithm.DISCRIMINATE
    gr, gs = _rows(got.batches)
    wr, _ = _rows(want.batches)
    assert gs.field(0).type == pa.date32() and gs.field(1).type == k_type
    assert [r[0] for r in gr] == [r[0] for r in wr]
    assert np.array_equal(np.array([r[1] for r in gr]).view(np.uint64), np.array([r[1] for r in wr]).view(np.uint64))
    # The dense algorithm takes integer keys only, as the reference's does.
    assert K.fold_dense(f, a_t, b_t) is None


def test_a_domain_carries_temporal_keys():
    a = _rel([pa.array([0, 1, 1], pa.int32()).cast(pa.date32()), pa.array([0, 0, 1]), pa.array([1.0, 2.0, 3.0])],
             ["i", "j", "v"])
    b = _rel([pa.array([0, 1]), pa.array([5, 5], pa.int64()).cast(pa.timestamp("s")), pa.array([10.0, 100.0])],
             ["j", "k", "v"])
    d = pa.record_batch([pa.array([1, 7, 0], pa.int32()).cast(pa.date32()),
                         pa.array([5, 5, 5], pa.int64()).cast(pa.timestamp("s"))], names=["i", "k"])
    got = K.fold(_fold(domain=True), a, b, K.Relation(d.schema, [d]))
    t = pa.Table.from_batches(got.batches)
    assert t.schema.field(0).type == pa.date32() and t.schema.field(1).type == pa.timestamp("s")
    rows = list(zip(t.column(0).cast(pa.int32()).to_pylist(), t.column(2).to_pylist()))
    assert rows == [(1, 2.0 * 10.0 + 3.0 * 100.0), (7, None), (0, 10.0)]


def test_unread_columns_of_any_type_and_unreadable_keys():
    i, j, va, j2, k, vb = _inputs(4)
    dec = pa.array([None] * len(i), pa.decimal128(20, 4))
    a_plus = _rel([pa.array(i), pa.array(j), pa.array(va), dec], ["i", "j", "v", "note"])
    a = _rel([pa.array(i), pa.array(j), pa.array(va)], ["i", "j", "v"])
    b = _rel([pa.array(j2), pa.array(k), pa.array(vb)], ["j", "k", "v"])
    f = _fold()
    got, _ = _rows(K.fold(f, a_plus, b).batches)
    want, _ = _rows(K.fold(f, a, b).batches)
    assert got == want
    # A decimal key: ranked by the host plan, so the fold declines.
    a_dec = _rel([pa.array([1, 2, 3], pa.int8()).cast(pa.decimal128(10, 2)), pa.array([0, 1, 2]), pa.array([1.0, 2.0, 3.0])],
                 ["i", "j", "v"])
    with pytest.raises(K.ArrowComputeError):
        K.fold(f, a_dec, b)
    assert "host plan" in K.last_call.message


def test_ranks_of_temporal_columns_are_their_values_ranks():
    rng = np.random.default_rng(5)
    x = rng.integers(-(1 << 50), 1 << 50, 20_000)
    x[::5] = x[1]
    for ty in (pa.timestamp("ns"), pa.duration("ms"), pa.date64()):
        col = pa.array(x, pa.int64()).cast(ty)
        bt = pa.record_batch([col], names=["c"])
        bi = pa.record_batch([pa.array(x)], names=["c"])
        got = K.rank_columns(K.Relation(bt.schema, [bt]), [0])
        want = K.rank_columns(K.Relation(bi.schema, [bi]), [0])
        assert np.array_equal(got.rank, want.rank) and np.array_equal(got.first, want.first)
