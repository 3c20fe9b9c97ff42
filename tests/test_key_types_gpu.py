"""Key types on the GPU path beyond integers, floats and strings: dates,
times, timestamps and durations rank, join and group as their values,
decimals of 32 to 256 bits as theirs and fixed-size binary as its bytes (the
reference ranks every type by Arrow's row format, keys.rs:16-37), and all
come back with their own types; the dense algorithm, which takes integer
keys only (dense.rs:93-110), declines them; a column of a type the library
can't read is allowed where no call reads it, and a key of such a type
declines to the host plan."""

import random

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


def _decimal(unscaled, t):
    # A decimal array of type t from its unscaled Python ints (None: NULL).
    w = t.byte_width
    data = b"".join((0 if v is None else v).to_bytes(w, "little", signed=True) for v in unscaled)
    valid = pa.array([v is not None for v in unscaled], pa.bool_()).buffers()[1]
    return pa.Array.from_buffers(t, len(unscaled), [valid, pa.py_buffer(data)],
                                 null_count=sum(v is None for v in unscaled))


def _unscaled(col):
    # A decimal column's unscaled values as Python ints (None: NULL).
    arr = col.combine_chunks() if isinstance(col, pa.ChunkedArray) else col
    w = arr.type.byte_width
    raw = arr.buffers()[1].to_pybytes() if len(arr) else b""
    return [int.from_bytes(raw[(arr.offset + i) * w:(arr.offset + i + 1) * w], "little", signed=True) if ok else None
            for i, ok in enumerate(arr.is_valid().to_pylist())]


def _as_int(col):
    # A temporal or decimal column's values as integers (32-bit temporal
    # types through int32).
    if pa.types.is_decimal(col.type):
        return _unscaled(col)
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
    note = pa.array([None] * len(i), pa.month_day_nano_interval())
    a_plus = _rel([pa.array(i), pa.array(j), pa.array(va), note], ["i", "j", "v", "note"])
    a = _rel([pa.array(i), pa.array(j), pa.array(va)], ["i", "j", "v"])
    b = _rel([pa.array(j2), pa.array(k), pa.array(vb)], ["j", "k", "v"])
    f = _fold()
    got, _ = _rows(K.fold(f, a_plus, b).batches)
    want, _ = _rows(K.fold(f, a, b).batches)
    assert got == want
    # An interval key: ranked by the host plan, so the fold declines.
    a_iv = _rel([pa.array([(1, 2, 3), (0, 0, 1), (1, 2, 3)], pa.month_day_nano_interval()), pa.array([0, 1, 2]),
                 pa.array([1.0, 2.0, 3.0])], ["i", "j", "v"])
    with pytest.raises(K.ArrowComputeError):
        K.fold(f, a_iv, b)
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


DECIMALS = [pa.decimal32(9, 2), pa.decimal64(18, 3), pa.decimal128(38, 4), pa.decimal256(76, 5)]


def _draw_unscaled(rng, n, precision):
    # Values over the type's whole range, small ones around zero, repeats
    # and NULLs.
    top = 10 ** precision - 1
    pool = [rng.randint(-top, top) for _ in range(n // 8)] + [0, 1, -1, top, -top]
    out = []
    for _ in range(n):
        r = rng.random()
        out.append(None if r < 0.05 else rng.randint(-50, 50) if r < 0.3 else rng.choice(pool) if r < 0.7
                   else rng.randint(-top, top))
    return out


def _rank_vs_oracle(columns):
    from oracle import oracle
    batch = pa.record_batch(list(columns), names=[f"c{i}" for i in range(len(columns))])
    got = K.rank_columns(K.Relation(batch.schema, [batch]), list(range(len(columns))))
    want = oracle.rank_columns(oracle.host_keys(list(columns), 0), batch.num_rows)
    assert np.array_equal(got.rank, want.rank) and np.array_equal(got.first, want.first)
    return got


@pytest.mark.parametrize("t", DECIMALS, ids=lambda t: f"decimal{t.bit_width}")
def test_ranks_of_decimal_columns_are_their_values_ranks(t):
    rng = random.Random(t.bit_width)
    vals = _draw_unscaled(rng, 6000, t.precision)
    got = _rank_vs_oracle([_decimal(vals, t)])
    # Ranks follow the values: NULL first, then ascending.
    order = sorted({v for v in vals if v is not None})
    assert len(got.first) == len(order) + (None in vals)
    firsts = [vals[r] for r in got.first]
    assert firsts == ([None] if None in vals else []) + order


def test_ranks_of_fixed_size_binary_and_mixed_wide_keys():
    rng = random.Random(7)
    n = 5000
    words = [bytes(rng.randrange(256) for _ in range(20)) for _ in range(300)]
    fsb = pa.array([None if rng.random() < 0.04 else rng.choice(words) for _ in range(n)], pa.binary(20))
    short = pa.array([bytes([rng.randrange(3), 0, rng.randrange(2)]) for _ in range(n)], pa.binary(3))
    d256 = _decimal([rng.choice([-(1 << 200), 0, 1 << 200, None, 5]) for _ in range(n)], pa.decimal256(76, 0))
    _rank_vs_oracle([fsb])
    _rank_vs_oracle([short, d256, fsb])
    _rank_vs_oracle([pa.array(rng.choices(range(4), k=n)), short, d256])
    # Dictionary-encoded decimals rank as their values.
    dvals = _draw_unscaled(rng, 40, 38)
    idx = [rng.randrange(len(dvals)) for _ in range(n)]
    dic = pa.DictionaryArray.from_arrays(pa.array(idx, pa.int16()), _decimal(dvals, pa.decimal128(38, 4)))
    plain = _decimal([dvals[x] for x in idx], pa.decimal128(38, 4))
    bd, bp = pa.record_batch([dic], names=["c"]), pa.record_batch([plain], names=["c"])
    got = K.rank_columns(K.Relation(bd.schema, [bd]), [0])
    want = K.rank_columns(K.Relation(bp.schema, [bp]), [0])
    assert np.array_equal(got.rank, want.rank) and np.array_equal(got.first, want.first)


@pytest.mark.parametrize("t", DECIMALS, ids=lambda t: f"decimal{t.bit_width}")
def test_decimal_keys_group_as_their_values(t):
    rng = np.random.default_rng(t.bit_width)
    n, m = 4000, 300
    i = rng.integers(-10 ** 8, 10 ** 8, 400)[rng.integers(0, 400, n)]
    j, j2 = rng.integers(0, 60, n), rng.integers(0, 60, m)
    k = rng.integers(-10 ** 8, 10 ** 8, m)
    k[::7] = k[3]
    va, vb = rng.normal(size=n), rng.normal(size=m)
    i_t = pa.decimal128(38, 4)
    a_d = _rel([_decimal([int(x) for x in i], i_t), pa.array(j), pa.array(va)], ["i", "j", "v"])
    b_d = _rel([pa.array(j2), _decimal([int(x) for x in k], t), pa.array(vb)], ["j", "k", "v"])
    a_i = _rel([pa.array(i), pa.array(j), pa.array(va)], ["i", "j", "v"])
    b_i = _rel([pa.array(j2), pa.array(k), pa.array(vb)], ["j", "k", "v"])
    f = _fold()
    got = K.fold(f, a_d, b_d)
    want = K.fold(f, a_i, b_i)
    assert got.algorithm == K.Algorithm.DISCRIMINATE
    gr, gs = _rows(got.batches)
    wr, _ = _rows(want.batches)
    assert gs.field(0).type == i_t and gs.field(1).type == t
    assert [r[0] for r in gr] == [r[0] for r in wr]
    assert np.array_equal(np.array([r[1] for r in gr]).view(np.uint64), np.array([r[1] for r in wr]).view(np.uint64))
    assert K.fold_dense(f, a_d, b_d) is None


def test_fixed_size_binary_and_dictionary_decimal_keys_in_a_fold():
    # Fixed-size binary orders as binary of one length does; a dictionary of
    # decimals groups as its values and comes back dictionary-encoded.
    rng = random.Random(11)
    n, m = 3000, 200
    words = [bytes(rng.randrange(256) for _ in range(12)) for _ in range(50)]
    i = [rng.choice(words) for _ in range(n)]
    j, j2 = [rng.randrange(40) for _ in range(n)], [rng.randrange(40) for _ in range(m)]
    kvals = _draw_unscaled(rng, 30, 38)
    kidx = [rng.randrange(len(kvals)) for _ in range(m)]
    va, vb = [rng.gauss(0, 1) for _ in range(n)], [rng.gauss(0, 1) for _ in range(m)]
    t = pa.decimal128(38, 4)
    kd = pa.DictionaryArray.from_arrays(pa.array(kidx, pa.int8()), _decimal(kvals, t))
    kp = _decimal([kvals[x] for x in kidx], t)
    f = _fold()
    got = K.fold(f, _rel([pa.array(i, pa.binary(12)), pa.array(j), pa.array(va)], ["i", "j", "v"]),
                 _rel([pa.array(j2), kd, pa.array(vb)], ["j", "k", "v"]))
    want = K.fold(f, _rel([pa.array(i, pa.binary()), pa.array(j), pa.array(va)], ["i", "j", "v"]),
                  _rel([pa.array(j2), kp, pa.array(vb)], ["j", "k", "v"]))
    tg, tw = pa.Table.from_batches(got.batches), pa.Table.from_batches(want.batches)
    assert tg.schema.field(0).type == pa.binary(12)
    assert pa.types.is_dictionary(tg.schema.field(1).type) and tg.schema.field(1).type.value_type == t
    assert tg.column(0).to_pylist() == tw.column(0).to_pylist()
    assert _unscaled(tg.column(1).combine_chunks().dictionary_decode()) == _unscaled(tw.column(1))
    assert np.array_equal(np.array(tg.column(2).to_pylist()).view(np.uint64),
                          np.array(tw.column(2).to_pylist()).view(np.uint64))
