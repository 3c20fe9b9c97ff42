"""Semantics the kernels must keep, on the GPU against the oracle:

- dense folds whose factors hold NaN, +-inf and -0.0, in a and in b
  (dense.rs:328-390, 658-700: such factors are never offered to a backend,
  the host's order of additions decides the result);
- budgets (crates/einfold-kernels/tests/kernels_vs_sql.rs:29-37): given
  exactly the bytes a call asked for with no limit, the same rows by the same
  algorithm, bit for bit; given one byte fewer, a memory error;
- the bounded device-side wait: a wait on an mbarrier nothing arrives on runs
  out, the call reports EINFOLD_TIMEOUT and the context stays usable;
- the softmax weights' exp (Tang's method) within 3 units in the last place
  of exp over [-708, 709] (2.17 the largest seen over 1.1e7 arguments), and
  equal to the math library's exp outside it.
"""
import ctypes
import math

import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import _lib, ir, kernels as K
from oracle import oracle
from tests.tables import U, assert_same_rows, complete, matmul_fold, rows_of, split_bound

pytestmark = pytest.mark.gpu

SPECIAL = np.array([np.nan, np.inf, -np.inf, -0.0, 0.0], dtype=np.float64)


def _sprinkle(values, rng, share):
    v = values.copy()
    for i in range(len(v)):
        if rng.chance(share):
            v[i] = SPECIAL[rng.below(len(SPECIAL))]
    return v


@pytest.mark.parametrize("where", ["a", "b", "both"])
@pytest.mark.parametrize("precision", [K.Precision.SPLIT, K.Precision.FP64])
def test_dense_folds_with_nan_infinities_and_signed_zeros(where, precision):
    rng = oracle.Rng.seeded(31, len(where))
    ni, nj, nk = 37, 53, 29
    av = rng.units(ni * nj) * 2 - 1
    bv = rng.units(nj * nk) * 2 - 1
    if where in ("a", "both"):
        av = _sprinkle(av, rng, 0.03)
    if where in ("b", "both"):
        bv = _sprinkle(bv, rng, 0.03)
    # A row of a and a column of b of -0.0 only: groups whose every term is
    # -0.0 (the reference's sums start at +0.0).
    av.reshape(ni, nj)[5] = -0.0
    bv.reshape(nj, nk)[:, 7] = -0.0
    sa, a = complete(["i", "j"], [ni, nj], av, rng)
    sb, b = complete(["j", "k"], [nj, nk], bv, rng)
    f = matmul_fold()
    want = oracle.fold(f, sa, a, sb, b, None, oracle.schema(f, [sa, sb]))
    got = K.fold(f, K.Relation(sa, a), K.Relation(sb, b), options=K.Options(precision=precision))
    assert want.algorithm == "dense" and got.algorithm == K.Algorithm.DENSE
    # Non-finite factors take the FP64 product in the reference's order in
    # both precisions: the reference's bits, NaNs, infinities and zeros' signs.
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)
    g = rows_of(got.batches).column(2).to_numpy(zero_copy_only=False)
    assert np.isnan(g).any() and np.isinf(g).any()


def test_dense_fold_of_only_finite_values_with_signed_zeros_in_the_split_form():
    rng = oracle.Rng.seeded(32, 0)
    ni, nj, nk = 40, 30, 20
    av = rng.units(ni * nj) * 2 - 1
    bv = rng.units(nj * nk) * 2 - 1
    av.reshape(ni, nj)[3] = -0.0
    bv.reshape(nj, nk)[::2, 4] = -0.0
    sa, a = complete(["i", "j"], [ni, nj], av, rng)
    sb, b = complete(["j", "k"], [nj, nk], bv, rng)
    f = matmul_fold()
    want = rows_of(oracle.fold(f, sa, a, sb, b, None, oracle.schema(f, [sa, sb])).batches)
    got = rows_of(K.fold(f, K.Relation(sa, a), K.Relation(sb, b)).batches)
    A, B = av.reshape(ni, nj), bv.reshape(nj, nk)
    tol = split_bound(nj, np.abs(A).max(1), np.abs(B).max(0)) + 2 * nj * U * (np.abs(A) @ np.abs(B))
    assert_same_rows(got, want, tol.reshape(-1))
    w = want.column(2).to_numpy(zero_copy_only=False)
    g = got.column(2).to_numpy(zero_copy_only=False)
    zero = w == 0
    assert np.array_equal(np.signbit(g[zero]), np.signbit(w[zero]))


class Limit(K.Budget):
    """A budget that counts what it gives, up to a limit (kernels_vs_sql.rs:663-683)."""

    def __init__(self, limit):
        self.limit = limit
        self.given = 0

    def grow(self, nbytes):
        if self.given + nbytes <= self.limit:
            self.given += nbytes
            return True
        return False

    def shrink(self, nbytes):
        self.given -= nbytes


def _budget_property(run):
    free = Limit(2 ** 62)
    base = run(free)
    asked = free.given
    assert asked > 0
    exact = Limit(asked)
    again = run(exact)
    assert again[0] == base[0]
    assert_same_rows(again[1], base[1], exact=True)
    with pytest.raises(K.ArrowMemoryError):
        run(Limit(asked - 1))
    return asked


def _fold_run(f, sa, a, sb, b, domain=None):
    def run(budget):
        r = K.fold(f, K.Relation(sa, a), K.Relation(sb, b),
                   K.Relation(domain[0].schema, domain) if domain else None, options=K.Options(budget=budget))
        return r.algorithm, rows_of(r.batches)
    return run


def test_budget_of_the_dense_fold():
    rng = oracle.Rng.seeded(33, 0)
    sa, a = complete(["i", "j"], [50, 40], rng.units(2000), rng)
    sb, b = complete(["j", "k"], [40, 30], rng.units(1200), rng)
    run = _fold_run(matmul_fold(), sa, a, sb, b)
    assert run(Limit(2 ** 62))[0] == K.Algorithm.DENSE
    _budget_property(run)


def test_budget_of_the_discrimination_fold():
    rng = oracle.Rng.seeded(34, 0)
    n = 3000
    a = [pa.record_batch([pa.array([f"{rng.below(500):016x}" for _ in range(n)]),
                          pa.array([rng.below(10 ** 9) for _ in range(n)], pa.int64()),
                          pa.array(list(rng.units(n)))], names=["i", "j", "v"])]
    b = [pa.record_batch([pa.array([a[0].column(1)[rng.below(n)].as_py() for _ in range(n)], pa.int64()),
                          pa.array([f"k{rng.below(300)}" for _ in range(n)]),
                          pa.array(list(rng.units(n)))], names=["j", "k", "v"])]
    run = _fold_run(matmul_fold(), a[0].schema, a, b[0].schema, b)
    assert run(Limit(2 ** 62))[0] == K.Algorithm.DISCRIMINATE
    _budget_property(run)


def test_budget_of_the_chain():
    rng = oracle.Rng.seeded(35, 0)
    tabs = [complete(["i", "j"], [30, 20], rng.units(600), rng),
            complete(["j", "k"], [20, 25], rng.units(500), rng),
            complete(["k", "l"], [25, 10], rng.units(250), rng)]
    E = ir.EQ
    f = ir.Fold([E, E, E, E], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2),
                               ir.Operand([(2, 0), (3, 1)], 2)], [ir.Output(0), ir.Output(3)])

    def run(budget):
        r = K.fold_chain(f, [K.Relation(s, b) for s, b in tabs], options=K.Options(budget=budget))
        assert r is not None
        return "chain", rows_of(r)
    _budget_property(run)


def test_a_bounded_wait_runs_out_and_the_context_stays_usable():
    lib = _lib.load()
    ctx = _lib.context(0)
    waited = ctypes.c_uint64(0)
    for limit in (20_000, 1_000_000):  # 20 us, 1 ms
        st = lib.einfold_check_wait(ctx, limit, ctypes.byref(waited))
        assert st == _lib.TIMEOUT
        assert limit <= waited.value < limit + 50_000_000
    assert lib.einfold_check_wait(ctx, 3_000_000_000, None) == _lib.INVALID  # above the kernels' 2 s
    # The context still computes.
    rng = oracle.Rng.seeded(36, 0)
    sa, a = complete(["i", "j"], [20, 30], rng.units(600), rng)
    sb, b = complete(["j", "k"], [30, 10], rng.units(300), rng)
    f = matmul_fold()
    want = oracle.fold(f, sa, a, sb, b, None, oracle.schema(f, [sa, sb]))
    got = K.fold(f, K.Relation(sa, a), K.Relation(sb, b), options=K.Options(precision=K.Precision.FP64))
    assert_same_rows(rows_of(got.batches), rows_of(want.batches), exact=True)


def _ulps(got, x):
    """|got - exp(x)| in units in the last place of exp(x), exp(x) in long double."""
    ref = np.exp(x.astype(np.longdouble))
    ulp = np.spacing(ref.astype(np.float64)).astype(np.longdouble)
    return np.abs(got.astype(np.longdouble) - ref) / ulp


def _exp_on_device(x, shift):
    import torch

    lib = _lib.load()
    tx = torch.from_numpy(x).cuda()
    ty = torch.empty_like(tx)
    torch.cuda.synchronize()
    assert lib.einfold_exp_weights(_lib.context(0), tx.data_ptr(), ty.data_ptr(), len(x), shift, None) == _lib.OK
    return ty.cpu().numpy(), torch.exp(tx).cpu().numpy()


def test_the_weights_exp_is_within_three_ulps_over_its_range():
    assert np.finfo(np.longdouble).nmant >= 63, "needs x87 long double for the reference"
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-708.0, 709.0, 10_000_000), rng.uniform(-1.0, 1.0, 1_000_000),
                        np.array([-708.0, 709.0, -707.9999999999999, 708.9999999999999, 0.0, -0.0,
                                  math.log(2) / 128, -math.log(2) / 128, 1e-300, -1e-300])])
    got, cuda = _exp_on_device(x, -1)
    err = _ulps(got, x)
    assert err.max() <= 3.0, (err.max(), x[np.argmax(err)])
    assert err.mean() <= 0.5
    # CUDA's exp on the same arguments, for scale.
    assert _ulps(cuda, x).max() <= 2.0
    # Outside [-708, 709] and for NaN: the math library's exp.
    out = np.array([-709.5, -745.0, -746.0, 709.8, 710.0, np.inf, -np.inf, np.nan])
    g, c = _exp_on_device(out, -1)
    assert np.array_equal(g.view(np.uint64), c.view(np.uint64))


@pytest.mark.parametrize("shift", [0, 46, 64])
def test_the_shifted_weights_are_powers_of_two_times_exp(shift):
    rng = np.random.default_rng(shift)
    x = np.concatenate([rng.uniform(-700.0, 0.0, 2_000_000), np.array([0.0, -700.0, -1e-12])])
    got, _ = _exp_on_device(x, shift)
    err = _ulps(np.ldexp(got, -shift), x)
    assert err.max() <= 3.0
    # Below -708 the argument is clamped: a weight under 2^(shift - 1021).
    low, _ = _exp_on_device(np.array([-800.0, -1e6]), shift)
    assert (low > 0).all() and (low <= 2.0 ** (shift - 1021)).all()
