"""The attention pipeline through the Arrow entry points beyond what the
reference's placement takes (fused.rs:624-664 declines any missing cell):

- ragged groups through einfold_pipeline: each batch's rows present from
  position 0 to its own length, against the oracle run on each group alone,
  and, at config 4's size (64 groups, d = 128, lengths log-uniform in
  [128, 8192], window |tq - tk| <= 512), bit for bit against the ragged
  device-array entry that the bench times, with a sample of groups against
  the oracle;
- einfold_pipeline_backward: the gradients of the result with respect to
  q, k and v from Arrow tables, against torch float64 autograd, complete
  and ragged.
"""
import math

import numpy as np
import pyarrow as pa
import pytest

from einfold_b200 import ir, kernels as K
from oracle import oracle
from tests.tables import rows_of

pytestmark = pytest.mark.gpu

E = ir.Dimension(ir.KeyEquality.EQUAL)
I, D, J, B, C = 0, 1, 2, 3, 4
GE, LE = ir.Comparison.GREATER_OR_EQUAL, ir.Comparison.LESS_OR_EQUAL


def _pipeline(window=None, causal=False, scale=None):
    """out(b, tq, c) = softmax over tk of SUM_d q.x * k.x, weighted v.x."""
    def operand(own):
        return ir.Operand([ir.Key(B, 0)] + [ir.Key(dd, i + 1) for i, dd in enumerate(own)], len(own) + 1)

    producer = ir.Fold([E, E, E, E], [operand([I, D]), operand([J, D])],
                       [ir.Output(B), ir.Output(I), ir.Output(J)])
    conds = []
    if window is not None:
        conds += [ir.Condition(I, GE, J, -window), ir.Condition(I, LE, J, window)]
    if causal:
        conds += [ir.Condition(I, GE, J, 0)]
    if conds:
        producer = producer.with_conditions(conds)
    values = ir.Operand([ir.Key(B, 0), ir.Key(J, 1), ir.Key(4, 2)], 3)
    weight = ir.Weight.exp() if scale is None else ir.Weight.exp(ir.Scale.times(scale))
    return ir.Pipeline(producer, weight, [E], values, [B, I, 4], ir.Normalizer.KEPT_GROUPS)


def _tables(Q, K_, V, lengths, batches=2):
    """q(b, t, d, x), k(b, t, d, x), v(b, t, c, x) from [b][t][..] arrays,
    batch b's rows for t < lengths[b] only, in shuffled batches."""
    rng = np.random.default_rng(3)

    def table(arr, names):
        nb, nt, nf = arr.shape
        b, t, f = np.indices(arr.shape).reshape(3, -1)
        keep = t < np.asarray(lengths)[b]
        order = rng.permutation(int(keep.sum()))
        cols = [pa.array(x[keep][order]) for x in (b, t, f)] + [pa.array(arr.reshape(-1)[keep][order])]
        tab = pa.Table.from_arrays(cols, names=names)
        n = tab.num_rows
        cuts = sorted(set([0, n] + list(rng.integers(0, n + 1, batches - 1))))
        return tab.schema, [tab.slice(lo, hi - lo).combine_chunks().to_batches()[0] if hi > lo else
                            tab.slice(0, 0).to_batches()[0] for lo, hi in zip(cuts[:-1], cuts[1:])]

    return table(Q, ["b", "t", "d", "x"]), table(K_, ["b", "t", "d", "x"]), table(V, ["b", "t", "c", "x"])


def _inputs(nb, lmax, d, c, seed):
    rng = np.random.default_rng(seed)
    return (rng.normal(0, 1 / math.sqrt(d), (nb, lmax, d)), rng.normal(0, 1 / math.sqrt(d), (nb, lmax, d)),
            rng.normal(0, 1, (nb, lmax, c)))


def _group_oracle(p, Q, K_, V, b, n):
    (sq, q), (sk, k), (sv, v) = _tables(Q[b:b + 1, :n], K_[b:b + 1, :n], V[b:b + 1, :n], [n], batches=1)
    out_schema = oracle.pipeline_schema(p, [sq, sk, sv])
    got = oracle.pipeline(p, q, k, v, out_schema, oracle.Options(threads=4))
    t = rows_of(got.batches)
    vals = t.column(3).to_numpy(zero_copy_only=False).reshape(n, -1)
    return vals


@pytest.mark.parametrize("window", [None, 5])
def test_ragged_groups_through_the_pipeline_entry(window):
    nb, lmax, d, c = 5, 70, 16, 3
    lengths = [70, 1, 33, 64, 65]
    Q, K_, V = _inputs(nb, lmax, d, c, 1)
    p = _pipeline(window)
    (sq, q), (sk, k), (sv, v) = _tables(Q, K_, V, lengths)
    got = K.pipeline(p, [K.Relation(sq, q), K.Relation(sk, k), K.Relation(sv, v)])
    assert got is not None, K.last_call.message
    t = rows_of(got.batches)
    assert t.num_rows == sum(lengths) * c
    bcol, tcol = t.column(0).to_numpy(), t.column(1).to_numpy()
    vals = t.column(3).to_numpy(zero_copy_only=False)
    at = 0
    for b, n in enumerate(lengths):
        rows = slice(at, at + n * c)
        assert (bcol[rows] == b).all() and np.array_equal(tcol[rows], np.repeat(np.arange(n), c))
        want = _group_oracle(p, Q, K_, V, b, n)
        assert np.abs(vals[rows].reshape(n, c) - want).max() <= 1e-12 * np.abs(V[b, :n]).max()
        at += n * c


def test_a_missing_cell_inside_a_group_still_declines():
    nb, lmax, d, c = 2, 20, 4, 2
    Q, K_, V = _inputs(nb, lmax, d, c, 2)
    (sq, q), (sk, k), (sv, v) = _tables(Q, K_, V, [20, 12])
    # Drop one k row in the middle of batch 1: not a prefix.
    kt = pa.Table.from_batches(k)
    keep = ~((kt.column(0).to_numpy() == 1) & (kt.column(1).to_numpy() == 5) & (kt.column(2).to_numpy() == 0))
    k2 = kt.filter(pa.array(keep)).to_batches()
    assert K.pipeline(_pipeline(), [K.Relation(sq, q), K.Relation(sk, k2), K.Relation(sv, v)]) is None
    # Lengths that differ between k and v decline too.
    (sv2, v2) = _tables(Q, K_, V, [20, 11])[2]
    assert K.pipeline(_pipeline(), [K.Relation(sq, q), K.Relation(sk, k), K.Relation(sv2, v2)]) is None


def _ragged_lengths(groups=64, lo=128, hi=8192, seed=0):
    from einfold_b200 import synthetic as S

    u = S.units(seed, 9, groups, device="cpu").double().numpy()
    return np.floor(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64)


def test_config_four_groups_from_arrow_tables():
    import torch

    from einfold_b200 import autograd as A

    lengths = _ragged_lengths()
    nb, d, c, window = 64, 128, 1, 512
    lmax = int(lengths.max())
    rng = np.random.default_rng(4)
    Q = rng.normal(0, 1 / math.sqrt(d), (nb, lmax, d))
    K_ = rng.normal(0, 1 / math.sqrt(d), (nb, lmax, d))
    V = rng.normal(0, 1 / math.sqrt(d), (nb, lmax, d))
    pos = np.arange(lmax)[None, :, None] < lengths[:, None, None]
    Q, K_, V = Q * pos, K_ * pos, V * pos
    p = _pipeline(window)
    (sq, q), (sk, k), (sv, v) = _tables(Q, K_, V, lengths)
    got = K.pipeline(p, [K.Relation(sq, q), K.Relation(sk, k), K.Relation(sv, v)])
    assert got is not None, K.last_call.message
    t = rows_of(got.batches)
    assert t.num_rows == int(lengths.sum()) * d
    vals = t.column(3).to_numpy(zero_copy_only=False)
    # The same bits as the ragged device-array entry on the padded arrays.
    tq, tk, tv = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (Q, K_, V))
    tl = torch.from_numpy(lengths).cuda()
    out, _ = A.attention_forward(tq, tk, tv, A.window(window), 1.0, K.Precision.SPLIT, q_lengths=tl, k_lengths=tl)
    dev = out.cpu().numpy()
    want = np.concatenate([dev[b, :lengths[b]].reshape(-1) for b in range(nb)])
    assert np.array_equal(vals.view(np.uint64), want.view(np.uint64))
    # A sample of groups against the oracle, each alone.
    starts = np.concatenate([[0], np.cumsum(lengths * d)])
    for b in (int(np.argmin(lengths)), 7, int(np.argmax(lengths))):
        n = int(lengths[b])
        w = _group_oracle(p, Q, K_, V, b, n)
        g = vals[starts[b]:starts[b + 1]].reshape(n, d)
        assert np.abs(g - w).max() <= 1e-12 * np.abs(V[b, :n]).max()


def _torch_grads(Q, K_, V, dO, lengths, window=None, causal=False, scale=1.0):
    import torch

    grads = []
    for b, n in enumerate(lengths):
        q, k, v = (torch.tensor(x[b, :n], dtype=torch.float64, requires_grad=True) for x in (Q, K_, V))
        s = scale * (q @ k.T)
        i = torch.arange(n)[:, None]
        j = torch.arange(n)[None, :]
        allowed = torch.ones(n, n, dtype=torch.bool)
        if window is not None:
            allowed &= (i - j).abs() <= window
        if causal:
            allowed &= i >= j
        out = torch.softmax(s.masked_fill(~allowed, float("-inf")), -1) @ v
        g = torch.autograd.grad(out, (q, k, v), torch.tensor(dO[b, :n]))
        grads.append([x.numpy() for x in g])
    return grads


def _d_out_table(dO, lengths):
    nb, lmax, c = dO.shape
    b, t, cc = np.indices(dO.shape).reshape(3, -1)
    keep = t < np.asarray(lengths)[b]
    return pa.record_batch([pa.array(b[keep]), pa.array(t[keep]), pa.array(cc[keep]),
                            pa.array(dO.reshape(-1)[keep])], names=["b", "t", "c", "g"])


@pytest.mark.parametrize("ragged,causal,scale", [(False, True, None), (True, False, 0.25), (True, True, None)])
def test_pipeline_backward_matches_torch(ragged, causal, scale):
    nb, lmax, d, c = 3, 150, 16, 8
    lengths = [150, 97, 150] if ragged else [150] * nb
    Q, K_, V = _inputs(nb, lmax, d, c, 5)
    dO = np.random.default_rng(6).normal(0, 1, (nb, lmax, c))
    window = 40 if ragged else None
    p = _pipeline(window, causal, scale)
    (sq, q), (sk, k), (sv, v) = _tables(Q, K_, V, lengths)
    dout = _d_out_table(dO, lengths)
    got = K.pipeline_backward(p, [K.Relation(sq, q), K.Relation(sk, k), K.Relation(sv, v)],
                              K.Relation(dout.schema, [dout]))
    assert got is not None, K.last_call.message
    want = _torch_grads(Q, K_, V, dO, lengths, window, causal, 1.0 if scale is None else scale)
    for which, width in ((0, d), (1, d), (2, c)):
        t = rows_of(got[which])
        assert t.column_names == ["b", "t", "d" if which < 2 else "c", "grad"]
        g = t.column(3).to_numpy(zero_copy_only=False)
        at = 0
        for b, n in enumerate(lengths):
            rows = slice(at, at + n * width)
            assert (t.column(0).to_numpy()[rows] == b).all()
            w = want[b][which]
            err = np.abs(g[rows].reshape(n, width) - w).max()
            assert err <= 1e-11 * max(np.abs(w).max(), 1e-300), (which, b, err)
            at += n * width
        assert at == t.num_rows


def test_pipeline_backward_of_a_missing_d_out_row_is_zero_and_others_decline():
    nb, lmax, d, c = 1, 40, 8, 2
    Q, K_, V = _inputs(nb, lmax, d, c, 7)
    dO = np.random.default_rng(8).normal(0, 1, (nb, lmax, c))
    p = _pipeline()
    (sq, q), (sk, k), (sv, v) = _tables(Q, K_, V, [lmax])
    ops = [K.Relation(sq, q), K.Relation(sk, k), K.Relation(sv, v)]
    dO[0, 10:] = 0.0
    full = _d_out_table(dO, [lmax])
    part = _d_out_table(dO[:, :10], [10])
    a = K.pipeline_backward(p, ops, K.Relation(full.schema, [full]))
    b = K.pipeline_backward(p, ops, K.Relation(part.schema, [part]))
    for x, y in zip(a, b):
        assert rows_of(x).equals(rows_of(y))
    # A sigmoid weight: not attention-shaped, declined.
    one = ir.Expression.literal(1.0)
    s = ir.Expression.column(0, 0)
    sig = one.binary(ir.Binary.DIVIDE, one.binary(ir.Binary.ADD, s.unary(ir.Unary.NEGATE).unary(ir.Unary.EXP)))
    p2 = ir.Pipeline(p.producer(), ir.Weight.of_expression(sig), [E], p.values(), [B, I, 4],
                     ir.Normalizer.KEPT_GROUPS)
    assert K.pipeline_backward(p2, ops, K.Relation(full.schema, [full])) is None


class _Ledger(K.Budget):
    """A budget that grants up to `cap` bytes at once and records what it was
    asked, granted and given back."""

    def __init__(self, cap):
        self.cap, self.out, self.peak, self.asked = cap, 0, 0, []

    def grow(self, n):
        self.asked.append(n)
        if self.out + n > self.cap:
            return False
        self.out += n
        self.peak = max(self.peak, self.out)
        return True

    def shrink(self, n):
        self.out -= n


def test_pipeline_backward_asks_the_budget_for_its_exports():
    # 4 causal batches of T = 1024, d = 64: about 8.3 MB of exports (P's digit
    # tiles and dS over the allowed tiles) a batch. With the whole granted,
    # one chunk; under 20 MB, two buffers of one batch each; with nothing
    # granted, the kernels that recompute the scores. Same bits every time,
    # and every granted byte given back.
    nb, lmax, d, c = 4, 1024, 64, 64
    Q, K_, V = _inputs(nb, lmax, d, c, 9)
    dO = np.random.default_rng(10).normal(0, 1, (nb, lmax, c))
    p = _pipeline(causal=True)
    (sq, q), (sk, k), (sv, v) = _tables(Q, K_, V, [lmax] * nb)
    dout = _d_out_table(dO, [lmax] * nb)
    ops = [K.Relation(sq, q), K.Relation(sk, k), K.Relation(sv, v)]

    def run(budget):
        got = K.pipeline_backward(p, ops, K.Relation(dout.schema, [dout]), K.Options(budget=budget))
        assert got is not None, K.last_call.message
        return [rows_of(g).column(3).to_numpy(zero_copy_only=False) for g in got]

    want = run(None)
    for cap, granted in ((1 << 40, True), (20 << 20, True), (0, False)):
        ledger = _Ledger(cap)
        got = run(ledger)
        for x, y in zip(got, want):
            assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), cap
        assert ledger.out == 0, (cap, ledger.out)
        assert ledger.asked, cap
        assert (ledger.peak > 0) == granted, (cap, ledger.peak)
        assert ledger.peak <= cap
        if cap == 20 << 20:
            assert ledger.peak > 8 << 20 and len(ledger.asked) > 1, ledger.asked
