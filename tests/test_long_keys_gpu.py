"""Keys of any length on the GPU: rank_columns (discriminate.rs:240-277, the
by_bytes branch at :165-209 for keys whose varying bytes don't fit a word)
and the discrimination fold over long or many-column keys, against the
oracle's restatement: the same ranks and first rows, the same result rows
bit for bit."""
import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests.tables import assert_same_rows, reference_facts, rows_of

pytestmark = pytest.mark.gpu

E = ir.Dimension(ir.KeyEquality.EQUAL)


def _rank_both(columns, float_keys=0):
    batch = pa.record_batch(list(columns), names=[f"c{i}" for i in range(len(columns))])
    got = K.rank_columns(K.Relation(batch.schema, [batch]), list(range(len(columns))), K.FloatKeys(float_keys))
    host = oracle.host_keys(list(columns), float_keys)
    want = oracle.rank_columns(host, batch.num_rows)
    assert np.array_equal(got.rank, want.rank)
    assert np.array_equal(got.first, want.first)
    return got


def test_keys_with_a_100000_byte_shared_prefix():
    # discriminate.rs:663-683: 200 keys sharing a 100,000-byte prefix, in
    # reverse order, sort as their bytes.
    lp = reference_facts()["long_prefix"]
    n = lp["keys"]
    prefix = lp["char"] * lp["prefix_bytes"]
    strings = [f"{prefix}{i:0{lp['digits']}}" for i in reversed(range(n))]
    got = _rank_both([pa.array(strings)])
    assert len(got.first) == n
    assert [strings[got.first[r]] for r in range(n)] == sorted(strings)
    assert np.array_equal(got.rank, np.arange(n - 1, -1, -1, dtype=np.uint32))


def test_long_strings_with_prefixes_zeros_and_nulls():
    rng = oracle.Rng.seeded(21, 0)
    stems = ["https://example.org/" + "a/" * 20, "https://example.org/" + "a/" * 19 + "b", "", "x" * 70]
    vals = []
    for _ in range(3000):
        r = rng.below(10)
        if r == 0:
            vals.append(None)
            continue
        s = stems[rng.below(len(stems))] + "".join(chr(97 + rng.below(3)) for _ in range(rng.below(6)))
        if r == 1:
            s += "\x00"  # a value and the same value with a zero after it differ
        vals.append(s)
    _rank_both([pa.array(vals)])
    _rank_both([pa.array([None if v is None else v.encode() for v in vals], pa.binary())])
    _rank_both([pa.array(vals, pa.large_string())])


@pytest.mark.parametrize("float_keys", [0, 1])
def test_many_columns_of_mixed_types(float_keys):
    rng = oracle.Rng.seeded(22, float_keys)
    n = 5000
    cols = [
        pa.array([f"{rng.below(2 ** 32):016x}" for _ in range(n)]),
        pa.array([None if rng.chance(0.05) else f"{rng.below(40):016x}" for _ in range(n)]),
        pa.array([rng.below(7) - 3 for _ in range(n)], pa.int64()),
        pa.array([[0.0, -0.0, 1.5, float("nan"), -2.0][rng.below(5)] for _ in range(n)], pa.float64()),
        pa.array([rng.below(3) for _ in range(n)], pa.int8()),
        pa.array([None if rng.chance(0.1) else rng.chance(0.5) for _ in range(n)], pa.bool_()),
    ]
    # Few distinct values per column but many together: keys of 6 columns,
    # about 50 bytes, with ties that only the later words break.
    for c in range(len(cols)):
        _rank_both(cols[: c + 1], float_keys)
    _rank_both(cols[1:], float_keys)


def test_more_than_eight_key_columns():
    rng = oracle.Rng.seeded(23, 0)
    n = 2000
    cols = [pa.array([rng.below(3) for _ in range(n)], pa.int32()) for _ in range(11)]
    got = _rank_both(cols)
    assert len(got.first) == len({tuple(c[i].as_py() for c in cols) for i in range(n)})


def test_all_keys_equal_and_empty_relations():
    _rank_both([pa.array(["q" * 100] * 50)])
    _rank_both([pa.array(["q" * 100] * 50), pa.array([7] * 50, pa.int64())])
    got = K.rank_columns(K.Relation(pa.schema([("c", pa.string())]),
                                    [pa.record_batch([pa.array([], pa.string())], names=["c"])]), [0])
    assert len(got.rank) == 0 and len(got.first) == 0


def _fold_both(f, a, b):
    sa, sb = a[0].schema, b[0].schema
    want = oracle.fold(f, sa, a, sb, b, None, oracle.schema(f, [sa, sb]))
    got = K.fold(f, K.Relation(sa, a), K.Relation(sb, b))
    return got, want


def test_fold_over_two_hex_string_columns_and_an_integer():
    # Output key x = (16-hex, 16-hex, int64): 19 + 19 + 9 bytes, beyond
    # four words; join key j a 63-bit hash; y one 16-hex string.
    rng = oracle.Rng.seeded(24, 0)
    n = 20_000
    hexes = [f"{rng.below(2 ** 63):016x}" for _ in range(300)]
    pool = [int(x) for x in rng.u64s(400) >> np.uint64(1)]
    a = [pa.record_batch([pa.array([hexes[rng.below(300)] for _ in range(n)]),
                          pa.array([hexes[rng.below(30)] for _ in range(n)]),
                          pa.array([rng.below(5) for _ in range(n)], pa.int64()),
                          pa.array([pool[rng.below(400)] for _ in range(n)], pa.int64()),
                          pa.array(list((rng.units(n) * 2 - 1)))], names=["i1", "i2", "i3", "j", "v"])]
    b = [pa.record_batch([pa.array([pool[rng.below(400)] for _ in range(n)], pa.int64()),
                          pa.array([hexes[rng.below(300)] for _ in range(n)]),
                          pa.array([None if rng.chance(0.02) else float(x) for x in (rng.units(n) * 2 - 1)])],
                         names=["j", "k", "v"])]
    f = ir.Fold([E, E, E, E, E], [ir.Operand([(0, 0), (1, 1), (2, 2), (3, 3)], 4),
                                  ir.Operand([(3, 0), (4, 1)], 2)],
                [ir.Output(0), ir.Output(1), ir.Output(2), ir.Output(4)])
    got, want = _fold_both(f, a, b)
    assert got.algorithm == K.Algorithm.DISCRIMINATE
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_fold_joined_on_long_url_keys():
    rng = oracle.Rng.seeded(25, 0)
    urls = [f"https://example.org/{'section/' * (1 + rng.below(12))}{rng.below(50)}" for _ in range(120)]
    n = 3000
    a = [pa.record_batch([pa.array([rng.below(40) for _ in range(n)], pa.int64()),
                          pa.array([urls[rng.below(120)] for _ in range(n)]),
                          pa.array(list(rng.units(n) * 2 - 1))], names=["i", "j", "v"])]
    b = [pa.record_batch([pa.array([urls[rng.below(120)] for _ in range(n)]),
                          pa.array([urls[rng.below(120)] for _ in range(n)]),
                          pa.array(list(rng.units(n) * 2 - 1))], names=["j", "k", "v"])]
    f = ir.Fold([E, E, E], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                [ir.Output(0), ir.Output(2)])
    got, want = _fold_both(f, a, b)
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_two_column_keys_beyond_4m_rows():
    # Keys of two int64 columns (more than one word) over 4.4M rows: the
    # ranks go back to rows by bucket (beyond L2's share), as the one-word
    # case does; the order of non-NULL integer keys is their signed
    # lexicographic order, checked against the oracle on a prefix of rows.
    n = 4_400_000
    rng = oracle.Rng.seeded(14, 2)
    c1 = (rng.u64s(n) % np.uint64(3000)).astype(np.int64) - 1500
    c2 = (rng.u64s(n) >> np.uint64(1)).astype(np.int64) * np.where(rng.u64s(n) & np.uint64(1), 1, -1)
    dup = np.arange(7, n, 7)  # every seventh row repeats an earlier row's key
    c1[dup], c2[dup] = c1[dup // 2], c2[dup // 2]
    batch = pa.record_batch([pa.array(c1), pa.array(c2)], names=["c0", "c1"])
    got = K.rank_columns(K.Relation(batch.schema, [batch]), [0, 1], K.FloatKeys(0))
    order = np.lexsort((c2, c1))
    s1, s2 = c1[order], c2[order]
    head = np.r_[True, (s1[1:] != s1[:-1]) | (s2[1:] != s2[:-1])]
    want_rank = np.empty(n, np.int64)
    want_rank[order] = np.cumsum(head) - 1
    assert np.array_equal(got.rank.astype(np.int64), want_rank)
    assert np.array_equal(got.first.astype(np.int64), order[head])
    m = 60_000
    small = _rank_both([pa.array(c1[:m]), pa.array(c2[:m])])
    o = np.lexsort((c2[:m], c1[:m]))
    h = np.r_[True, (c1[:m][o][1:] != c1[:m][o][:-1]) | (c2[:m][o][1:] != c2[:m][o][:-1])]
    assert np.array_equal(small.first.astype(np.int64), o[h])
