"""The discrimination fold on the GPU against the oracle (discriminate.rs
restated): same rows in the same order, same NULLs, and the same bits, as
every group's terms are added in the reference's order."""
import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests.tables import assert_same_rows, complete, matmul_fold, rows_of

pytestmark = pytest.mark.gpu

E, ND = ir.Dimension(ir.KeyEquality.EQUAL), ir.Dimension(ir.KeyEquality.NOT_DISTINCT)


def _both(f, a, b, domain=None, options=None, float_keys=0):
    sa, sb = a[0].schema, b[0].schema
    out_schema = oracle.schema(f, [sa, sb], domain[0].schema if domain else None)
    want = oracle.fold(f, sa, a, sb, b, domain, out_schema, oracle.Options(float_keys=float_keys))
    opts = options or K.Options(host=K.Host(K.FloatKeys(float_keys)))
    got = K.fold(f, K.Relation(sa, a), K.Relation(sb, b),
                 K.Relation(domain[0].schema, domain) if domain else None, options=opts)
    return got, want


def test_nulls_in_b_send_the_matmul_fold_to_discrimination():
    # The 512 x 512 . 512 x 256 fold's shape, scaled: 1% of b's factors NULL.
    rng = oracle.Rng.seeded(0, 0x5eedf01d)
    ni, nj, nk = 64, 64, 32
    sa, a = complete(["i", "j"], [ni, nj], rng.units(ni * nj) * 2 - 1, rng)
    bn = rng.units(nj * nk) < 0.01
    bn[3] = True
    sb, b = complete(["j", "k"], [nj, nk], rng.units(nj * nk) * 2 - 1, rng, nulls=bn)
    got, want = _both(matmul_fold(), a, b)
    assert want.algorithm == "discriminate" and got.algorithm == K.Algorithm.DISCRIMINATE
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_config_one_at_full_size():
    rng = oracle.Rng.seeded(0, 1)
    ni, nj, nk = 512, 512, 256
    sa, a = complete(["i", "j"], [ni, nj], rng.units(ni * nj) * 2 - 1, rng, batches=4)
    sb, b = complete(["j", "k"], [nj, nk], rng.units(nj * nk) * 2 - 1, rng, nulls=rng.units(nj * nk) < 0.01,
                     batches=4)
    got, want = _both(matmul_fold(), a, b)
    assert got.algorithm == K.Algorithm.DISCRIMINATE
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_duplicate_rows_count_twice():
    a = [pa.record_batch([pa.array([0, 0, 1, 1, 1]), pa.array([5, 5, 5, 6, 6]), pa.array([1.0, 2.0, 3.0, 4.0, None])],
                         names=["i", "j", "v"])]
    b = [pa.record_batch([pa.array([5, 5, 6]), pa.array([7, 7, 8]), pa.array([0.5, 0.25, -1.0])], names=["j", "k", "v"])]
    got, want = _both(matmul_fold(), a, b)
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def _keyed(keys_a, ja, va, jb, keys_b, vb, ta=pa.string(), tj=pa.int64(), tb=pa.string()):
    a = [pa.record_batch([pa.array(keys_a, ta), pa.array(ja, tj), pa.array(va, pa.float64())], names=["i", "j", "v"])]
    b = [pa.record_batch([pa.array(jb, tj), pa.array(keys_b, tb), pa.array(vb, pa.float64())], names=["j", "k", "v"])]
    return a, b


def test_string_keys_sort_as_bytes_and_null_groups():
    rng = oracle.Rng.seeded(3, 0)
    words = ["", "a", "ab", "b", "ba", "a\x00", "zz", None, "é", "abc"]
    n = 400
    ia = [words[rng.below(len(words))] for _ in range(n)]
    ja = [rng.below(20) for _ in range(n)]
    va = list(rng.units(n) * 2 - 1)
    jb = [rng.below(20) for _ in range(n)]
    kb = [words[rng.below(len(words))] for _ in range(n)]
    vb = [None if rng.chance(0.05) else float(x) for x in rng.units(n) * 2 - 1]
    a, b = _keyed(ia, ja, va, jb, kb, vb)
    got, want = _both(matmul_fold(), a, b)
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_string_keys_kept_in_hbm_match_the_host_result():
    # Results left in device memory keep string keys there too: the offsets
    # and bytes read back through DeviceBatch.strings equal the host result.
    rng = oracle.Rng.seeded(7, 0)
    words = ["", "a", "ab", "0123456789abcdef", "fedcba9876543210", "é", "abc", "zz"]
    n = 300
    ia = [words[rng.below(len(words))] for _ in range(n)]
    ja = [rng.below(15) for _ in range(n)]
    jb = [rng.below(15) for _ in range(n)]
    kb = [words[rng.below(len(words))] for _ in range(n)]
    a, b = _keyed(ia, ja, list(rng.units(n)), jb, kb, list(rng.units(n)))
    f = matmul_fold()
    ra, rb = K.Relation(a[0].schema, a), K.Relation(b[0].schema, b)
    host = rows_of(K.fold(f, ra, rb).batches)
    dev = K.fold(f, ra, rb, options=K.Options(result_on_device=True)).batches[0]
    try:
        assert dev.rows == host.num_rows
        for i in (0, 1):
            offsets, data = dev.strings(i)
            o, d = offsets.cpu().numpy(), bytes(data.cpu().numpy())
            got = [d[o[r]:o[r + 1]].decode() for r in range(dev.rows)]
            assert got == host.column(i).to_pylist()
        assert np.array_equal(dev.column(2).cpu().numpy(), host.column(2).to_numpy())
        with pytest.raises(TypeError):
            dev.column(0)
    finally:
        dev.release()


@pytest.mark.parametrize("equality", [E, ND])
def test_null_join_keys_under_either_equality(equality):
    rng = oracle.Rng.seeded(4, 0)
    n = 300
    ja = [None if rng.chance(0.1) else rng.below(12) for _ in range(n)]
    jb = [None if rng.chance(0.1) else rng.below(12) for _ in range(n)]
    a, b = _keyed([rng.below(9) for _ in range(n)], ja, list(rng.units(n)), jb, [rng.below(7) for _ in range(n)],
                  list(rng.units(n)), ta=pa.int32(), tb=pa.int16())
    f = ir.Fold([E, equality, E], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                [ir.Output(0), ir.Output(2)])
    got, want = _both(f, a, b)
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


@pytest.mark.parametrize("float_keys", [0, 1])
def test_signed_zero_float_keys(float_keys):
    ia = [0.0, -0.0, 1.5, -0.0, float("nan"), 2.0]
    ja = [1, 1, 1, 2, 2, 2]
    jb = [1, 2, 2]
    kb = [-0.0, 0.0, 3.0]
    a, b = _keyed(ia, ja, [1.0, 2.0, 3.0, 4.0, 5.0, 6.0], jb, kb, [10.0, 100.0, 1000.0], ta=pa.float64(),
                  tb=pa.float64())
    got, want = _both(matmul_fold(), a, b, float_keys=float_keys)
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_multi_column_keys_and_a_sparse_summed_dimension():
    rng = oracle.Rng.seeded(5, 0)
    n = 2000
    a = [pa.record_batch([pa.array([rng.below(5) for _ in range(n)], pa.int64()),
                          pa.array([f"s{rng.below(4)}" for _ in range(n)]),
                          pa.array([rng.below(10 ** 6) * 977 for _ in range(n)], pa.int64()),
                          pa.array(list(rng.units(n)))], names=["i1", "i2", "j", "v"])]
    b = [pa.record_batch([pa.array([rng.below(10 ** 6) * 977 if rng.chance(0.5) else a[0].column(2)[rng.below(n)].as_py()
                                    for _ in range(n)], pa.int64()),
                          pa.array([rng.below(6) for _ in range(n)], pa.uint32()),
                          pa.array(list(rng.units(n)))], names=["j", "k", "v"])]
    f = ir.Fold([E, E, E, E], [ir.Operand([(0, 0), (1, 1), (2, 2)], 3), ir.Operand([(2, 0), (3, 1)], 2)],
                [ir.Output(0), ir.Output(1), ir.Output(3)])
    got, want = _both(f, a, b)
    assert got.algorithm == K.Algorithm.DISCRIMINATE
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_a_domain_with_null_and_missing_keys():
    rng = oracle.Rng.seeded(6, 0)
    n = 500
    a, b = _keyed([rng.below(9) for _ in range(n)], [rng.below(15) for _ in range(n)], list(rng.units(n)),
                  [rng.below(15) for _ in range(n)], [rng.below(7) for _ in range(n)], list(rng.units(n)),
                  ta=pa.int64(), tb=pa.int64())
    dom = [pa.record_batch([pa.array([None if rng.chance(0.1) else rng.below(11) for _ in range(300)], pa.int64()),
                            pa.array([rng.below(9) for _ in range(300)], pa.int64()),
                            pa.array([f"row{r}" for r in range(300)])], names=["i", "k", "tag"])]
    for missing in (None, 0.0, -1.5):
        for eq in (ir.KeyEquality.EQUAL, ir.KeyEquality.NOT_DISTINCT):
            f = ir.Fold([E, E, E], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                        [ir.Output(0, ir.DomainKey(0, eq)), ir.Output(2, ir.DomainKey(1, eq))],
                        domain=ir.Domain((2, 0), missing))
            got, want = _both(f, a + [a[0].slice(0, 3)], b, dom)  # a duplicate: the dense algorithm declines
            assert got.algorithm == K.Algorithm.DISCRIMINATE
            assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_cross_join_and_empty_inputs():
    a = [pa.record_batch([pa.array([1, 2, 2], pa.int64()), pa.array([0.5, 1.5, 2.5])], names=["i", "v"])]
    b = [pa.record_batch([pa.array([7, 8], pa.int64()), pa.array([2.0, 4.0])], names=["k", "v"])]
    f = ir.Fold([E, E], [ir.Operand([(0, 0)], 1), ir.Operand([(1, 0)], 1)], [ir.Output(0), ir.Output(1)])
    got, want = _both(f, a, b)
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)
    empty_a = [a[0].slice(0, 0)]
    got, want = _both(f, empty_a, b)
    assert rows_of(got.batches).num_rows == 0 == rows_of(want.batches).num_rows
