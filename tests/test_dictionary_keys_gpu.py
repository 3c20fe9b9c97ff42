"""Dictionary-encoded key columns on the GPU path: they rank, join and group
as the plain columns of their values (a row is NULL where its index or its
dictionary value is), results carry them dictionary-encoded, and float
dictionaries compare by their bits whatever the host's float keys
(options.rs:19-22: DataFusion takes -0.0 and 0.0 as one key in float
columns, not in dictionary-encoded ones)."""
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
                   domain=ir.Domain((0, 1), 0.0) if domain else None)


def _dict(values, index, index_type=pa.int32(), value_type=pa.string()):
    idx = pa.array(index, type=index_type)
    return pa.DictionaryArray.from_arrays(idx, pa.array(values, type=value_type))


def _rows(batches):
    t = pa.Table.from_batches(batches)
    cols = []
    for c in t.columns:
        c = c.combine_chunks()
        cols.append(c.dictionary_decode() if pa.types.is_dictionary(c.type) else c)
    keys = list(zip(*[c.to_pylist() for c in cols[:-1]]))
    vals = np.asarray(cols[-1].fill_null(np.nan).to_numpy(zero_copy_only=False), np.float64)
    order = sorted(range(len(keys)), key=lambda r: tuple((k is None, k) for k in keys[r]))
    return [keys[r] for r in order], vals[order], t.schema


def _batches(arrays, names):
    # Two batches, with dictionaries of their own.
    n = len(arrays[0])
    h = n // 2
    return [pa.record_batch([a.slice(0, h) for a in arrays], names=names),
            pa.record_batch([a.slice(h) for a in arrays], names=names)]


def _split(batches):
    return batches[0].schema, batches


def test_dictionary_keys_fold_as_their_values():
    rng = np.random.default_rng(1)
    n = 3000
    words = [f"w{i:03}" for i in range(40)] + [None]  # a NULL dictionary value
    ia = rng.integers(0, len(words), n)
    ja = rng.integers(0, 50, n)
    null_index = rng.random(n) < 0.03
    i_dict = pa.DictionaryArray.from_arrays(pa.array(ia, type=pa.int32(), mask=null_index), pa.array(words))
    i_plain = pa.array([None if (m or words[x] is None) else words[x] for x, m in zip(ia, null_index)])
    kb = rng.integers(0, 30, 60)
    jb = rng.integers(0, 50, 60)
    k_vals = [f"k{i}" for i in range(30)]
    k_dict = _dict(k_vals, kb, pa.int8())
    k_plain = pa.array([k_vals[x] for x in kb])
    va, vb = pa.array(rng.normal(size=n)), pa.array(rng.normal(size=60))
    f = _fold()

    def rel(arrays, names):
        return K.Relation(*_split(_batches(arrays, names)))

    got = K.fold(f, rel([i_dict, pa.array(ja), va], ["i", "j", "v"]), rel([pa.array(jb), k_dict, vb], ["j", "k", "v"]))
    want = K.fold(f, rel([i_plain, pa.array(ja), va], ["i", "j", "v"]), rel([pa.array(jb), k_plain, vb], ["j", "k", "v"]))
    assert got.algorithm == want.algorithm == K.Algorithm.DISCRIMINATE
    gk, gv, gs = _rows(got.batches)
    wk, wv, _ = _rows(want.batches)
    assert pa.types.is_dictionary(gs.field(0).type) and pa.types.is_dictionary(gs.field(1).type)
    assert gs.field(1).type.index_type == pa.int8()
    assert gk == wk and any(k[0] is None for k in gk)
    assert np.array_equal(gv.view(np.uint64), wv.view(np.uint64))


def test_float_dictionaries_compare_by_bits():
    # Group by a float key holding 0.0 and -0.0 under SignedZerosEqual: one
    # group shown as 0.0 for the plain column, two for the dictionary.
    keys = [0.0, -0.0, 0.0, 2.5, -0.0]
    j = [0, 0, 1, 1, 0]
    v = [1.0, 2.0, 3.0, 4.0, 5.0]
    b = pa.record_batch([pa.array([0, 1]), pa.array([7, 7]), pa.array([1.0, 10.0])], names=["j", "k", "v"])
    f = _fold()
    host = K.Options(host=K.Host(K.FloatKeys.SIGNED_ZEROS_EQUAL))
    plain = pa.record_batch([pa.array(keys), pa.array(j), pa.array(v)], names=["i", "j", "v"])
    dic = pa.record_batch([_dict([0.0, -0.0, 2.5], [0, 1, 0, 2, 1], value_type=pa.float64()), pa.array(j),
                           pa.array(v)], names=["i", "j", "v"])
    gp = K.fold(f, K.Relation(plain.schema, [plain]), K.Relation(b.schema, [b]), options=host)
    gd = K.fold(f, K.Relation(dic.schema, [dic]), K.Relation(b.schema, [b]), options=host)
    pk, pv, _ = _rows(gp.batches)
    dk, dv, ds = _rows(gd.batches)
    assert pa.types.is_dictionary(ds.field(0).type)
    shown = lambda ks: sorted((np.float64(k[0]).view(np.uint64).item(), k[1]) for k in ks)  # noqa: E731
    assert shown(pk) == sorted([(np.float64(0.0).view(np.uint64).item(), 7), (np.float64(2.5).view(np.uint64).item(), 7)])
    assert len(dk) == 3 and {np.float64(k[0]).view(np.uint64).item() for k in dk} == {
        np.float64(x).view(np.uint64).item() for x in (0.0, -0.0, 2.5)}
    assert sorted(pv) == sorted([1.0 + 3.0 * 10.0 + 2.0 + 5.0, 40.0])
    assert sorted(dv) == sorted([1.0 + 30.0, 2.0 + 5.0, 40.0])


def test_a_domain_carries_its_dictionary_keys():
    a = pa.record_batch([_dict(["x", "y"], [0, 1, 1]), pa.array([0, 0, 1]), pa.array([1.0, 2.0, 3.0])],
                        names=["i", "j", "v"])
    b = pa.record_batch([pa.array([0, 1]), _dict(["p"], [0, 0]), pa.array([10.0, 100.0])], names=["j", "k", "v"])
    d = pa.record_batch([_dict(["y", "z", "x", None], [0, 1, 2, 3]), _dict(["p"], [0, 0, 0, 0])], names=["i", "k"])
    got = K.fold(_fold(domain=True), K.Relation(a.schema, [a]), K.Relation(b.schema, [b]), K.Relation(d.schema, [d]))
    t = pa.Table.from_batches(got.batches)
    assert pa.types.is_dictionary(t.schema.field(0).type)
    rows = list(zip(t.column(0).combine_chunks().dictionary_decode().to_pylist(),
                    t.column(1).combine_chunks().dictionary_decode().to_pylist(), t.column(2).to_pylist()))
    assert rows == [("y", "p", 2.0 * 10.0 + 3.0 * 100.0), ("z", "p", 0.0), ("x", "p", 10.0), (None, "p", 0.0)]


def test_ranks_of_a_dictionary_column_are_its_values_ranks():
    rng = np.random.default_rng(2)
    words = [f"s{i}" for i in rng.permutation(200)] + [None]
    idx = rng.integers(0, len(words), 5000)
    dic = _dict(words, idx)
    plain = pa.array([words[x] for x in idx])
    bd = pa.record_batch([dic], names=["c"])
    bp = pa.record_batch([plain], names=["c"])
    got = K.rank_columns(K.Relation(bd.schema, [bd]), [0])
    want = K.rank_columns(K.Relation(bp.schema, [bp]), [0])
    assert np.array_equal(got.rank, want.rank) and np.array_equal(got.first, want.first)
