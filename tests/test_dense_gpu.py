"""The dense fold on the GPU against the oracle (dense.rs restated)."""
import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests.tables import U, assert_same_rows, complete, matmul_fold, rows_of, split_bound

pytestmark = pytest.mark.gpu


def _matmul_case(seed, ni, nj, nk, a_null=0.0, key_type=pa.int64(), batches=3):
    rng = oracle.Rng.seeded(seed, 0x5eedf01d)
    av = rng.units(ni * nj) * 2 - 1
    bv = rng.units(nj * nk) * 2 - 1
    an = rng.units(ni * nj) < a_null if a_null else None
    sa, a = complete(["i", "j"], [ni, nj], av, rng, key_type, an, batches)
    sb, b = complete(["j", "k"], [nj, nk], bv, rng, key_type, None, batches)
    return (sa, a, sb, b, av.reshape(ni, nj), bv.reshape(nj, nk), an)


@pytest.mark.parametrize("shape", [(5, 7, 3), (64, 100, 48), (257, 129, 200), (512, 512, 256)])
def test_matmul_fold_split_matches_oracle(shape):
    ni, nj, nk = shape
    sa, a, sb, b, A, B, _ = _matmul_case(1, ni, nj, nk)
    f = matmul_fold()
    out_schema = oracle.schema(f, [sa, sb])
    want = oracle.fold(f, sa, a, sb, b, None, out_schema)
    got = K.fold(f, K.Relation(sa, a), K.Relation(sb, b))
    assert want.algorithm == "dense" and got.algorithm == K.Algorithm.DENSE
    terms = np.abs(A) @ np.abs(B)
    tol = split_bound(nj, np.abs(A).max(1), np.abs(B).max(0)) + 2 * nj * U * terms
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), tol.reshape(-1))


@pytest.mark.parametrize("shape", [(5, 7, 3), (64, 100, 48), (70, 5000, 30)])
def test_matmul_fold_fp64_is_the_references_bits(shape):
    ni, nj, nk = shape
    sa, a, sb, b, A, B, _ = _matmul_case(2, ni, nj, nk, a_null=0.1)
    f = matmul_fold()
    out_schema = oracle.schema(f, [sa, sb])
    want = oracle.fold(f, sa, a, sb, b, None, out_schema)
    got = K.fold(f, K.Relation(sa, a), K.Relation(sb, b), options=K.Options(precision=K.Precision.FP64))
    assert want.algorithm == "dense"
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def test_nulls_in_a_give_null_groups_and_the_same_values():
    ni, nj, nk = 40, 6, 9
    rng = oracle.Rng.seeded(3, 1)
    av = rng.units(ni * nj) * 2 - 1
    nulls = np.zeros(ni * nj, bool)
    nulls[:nj] = True  # row i = 0: every factor NULL, so its groups are NULL
    nulls[nj + 2] = True
    sa, a = complete(["i", "j"], [ni, nj], av, rng, nulls=nulls)
    sb, b = complete(["j", "k"], [nj, nk], rng.units(nj * nk), rng)
    f = matmul_fold()
    out_schema = oracle.schema(f, [sa, sb])
    want = oracle.fold(f, sa, a, sb, b, None, out_schema)
    got = K.fold(f, K.Relation(sa, a), K.Relation(sb, b))
    t = rows_of(got.batches)
    assert t.column(2).null_count == nk
    assert_same_rows(t, rows_of(want.batches), np.full(t.num_rows, 1e-13))


@pytest.mark.parametrize("key_type", [pa.int32(), pa.uint16(), pa.int8(), pa.uint64()])
def test_key_types_give_the_same_bits(key_type):
    sa, a, sb, b, *_ = _matmul_case(4, 20, 30, 10, key_type=key_type)
    sa64, a64, sb64, b64, *_ = _matmul_case(4, 20, 30, 10)
    f = matmul_fold()
    got = rows_of(K.fold(f, K.Relation(sa, a), K.Relation(sb, b)).batches)
    ref = rows_of(K.fold(f, K.Relation(sa64, a64), K.Relation(sb64, b64)).batches)
    assert got.column(0).type == key_type
    g = np.asarray(got.column(2).to_numpy(), np.float64).view(np.uint64)
    r = np.asarray(ref.column(2).to_numpy(), np.float64).view(np.uint64)
    assert np.array_equal(g, r)


def test_same_bits_on_any_batching():
    outs = []
    for batches in (1, 2, 7):
        sa, a, sb, b, *_ = _matmul_case(5, 33, 65, 17, batches=batches)
        outs.append(rows_of(K.fold(matmul_fold(), K.Relation(sa, a), K.Relation(sb, b)).batches))
    for t in outs[1:]:
        assert t.equals(outs[0])


def test_duplicates_decline_the_dense_algorithm():
    sa, a, sb, b, *_ = _matmul_case(6, 8, 8, 8)
    a = a + [a[0].slice(0, 1)]
    assert K.fold_dense(matmul_fold(), K.Relation(sa, a), K.Relation(sb, b)) is None


def test_holes_in_b_decline_without_a_zero_default():
    sa, a, sb, b, *_ = _matmul_case(7, 8, 8, 8)
    b = [bb.slice(1) if i == 0 else bb for i, bb in enumerate(b)]
    assert K.fold_dense(matmul_fold(), K.Relation(sa, a), K.Relation(sb, b)) is None


def test_a_domain_with_a_zero_default_takes_holes():
    rng = oracle.Rng.seeded(8, 0)
    ni, nj, nk = 12, 9, 7
    sa, a = complete(["i", "j"], [ni, nj], rng.units(ni * nj), rng)
    sb, b = complete(["j", "k"], [nj, nk], rng.units(nj * nk), rng)
    b = [bb.slice(2) if i == 0 else bb for i, bb in enumerate(b)]
    keys_i = [rng.below(ni + 2) for _ in range(200)]
    keys_k = [rng.below(nk + 2) for _ in range(200)]
    dom = pa.record_batch([pa.array(keys_i, pa.int64()), pa.array(keys_k, pa.int64())], names=["i", "k"])
    f = matmul_fold(domain=True, missing=0.0)
    out_schema = oracle.schema(f, [sa, sb], dom.schema)
    want = oracle.dense_fold(f, a, b, [dom], out_schema)
    got = K.fold_dense(f, K.Relation(sa, a), K.Relation(sb, b), K.Relation(dom.schema, [dom]))
    assert want is not None and got is not None
    assert_same_rows(rows_of(got), rows_of(want), np.full(200, 1e-13))


def test_unique_domain_keys_are_checked():
    rng = oracle.Rng.seeded(9, 0)
    sa, a = complete(["i", "j"], [4, 3], rng.units(12), rng)
    sb, b = complete(["j", "k"], [3, 5], rng.units(15), rng)
    dom = pa.record_batch([pa.array([0, 1, 1], pa.int64()), pa.array([0, 2, 2], pa.int64())], names=["i", "k"])
    f = matmul_fold(domain=True, missing=None)
    opts = K.Options(domain_rows=K.DomainRows.UNIQUE_KEYS)
    assert K.fold_dense(f, K.Relation(sa, a), K.Relation(sb, b), K.Relation(dom.schema, [dom]), options=opts) is None
    dom2 = pa.record_batch([pa.array([0, 1, 3], pa.int64()), pa.array([0, 2, 2], pa.int64())], names=["i", "k"])
    assert K.fold_dense(f, K.Relation(sa, a), K.Relation(sb, b), K.Relation(dom2.schema, [dom2]),
                        options=opts) is not None


def test_masked_groups_are_dropped():
    rng = oracle.Rng.seeded(10, 0)
    n, d = 20, 4
    sa, a = complete(["i", "j"], [n, d], rng.units(n * d), rng)
    sb, b = complete(["j", "k"], [d, n], rng.units(n * d), rng)
    f = matmul_fold().with_conditions([ir.Condition(0, ir.Comparison.GREATER_OR_EQUAL, 2, 0)])
    out_schema = oracle.schema(f, [sa, sb])
    want = oracle.dense_fold(f, a, b, None, out_schema)
    got = K.fold_dense(f, K.Relation(sa, a), K.Relation(sb, b))
    assert rows_of(got).num_rows == n * (n + 1) // 2
    assert_same_rows(rows_of(got), rows_of(want), np.full(n * (n + 1) // 2, split_bound(d, [1.0], [1.0])[0, 0]))


def test_device_relations_and_device_results_match_host_ones():
    import torch

    rng = oracle.Rng.seeded(11, 0)
    ni, nj, nk = 100, 64, 70
    sa, a = complete(["i", "j"], [ni, nj], rng.units(ni * nj) * 2 - 1, rng, batches=1, shuffle=False)
    sb, b = complete(["j", "k"], [nj, nk], rng.units(nj * nk) * 2 - 1, rng, batches=1, shuffle=False)
    f = matmul_fold()
    host = rows_of(K.fold(f, K.Relation(sa, a), K.Relation(sb, b)).batches)
    cols = lambda t: [torch.as_tensor(np.asarray(c.to_numpy())).cuda() for c in pa.Table.from_batches(t).columns]
    da = K.DeviceRelation(sa, cols(a))
    db = K.DeviceRelation(sb, cols(b))
    dev = K.fold(f, da, db, options=K.Options(result_on_device=True)).batches[0]
    assert dev.rows == host.num_rows
    for c in range(3):
        got = dev.column(c).cpu().numpy()
        want = np.asarray(host.column(c).to_numpy())
        assert np.array_equal(got.view(np.uint64) if got.dtype == np.float64 else got,
                              want.view(np.uint64) if want.dtype == np.float64 else want)
    dev.release()
