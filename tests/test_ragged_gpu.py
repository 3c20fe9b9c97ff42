"""Ragged batches (groups of different lengths in one call, padded to the
longest): each group against the same group run alone as a full batch,
against torch float64, and the padding rows' gradients zero, in both forms.
The split form gives the same bits as alone (the same digits, tiles and
integer sums); the FP64 form's online softmax takes its key tiles at
multiples of 64 in the padded layout, so there the rounding may differ."""
import pytest
import torch

from einfold_b200 import autograd as A
from einfold_b200.kernels import Precision
from tests.test_autograd_gpu import _reference

pytestmark = pytest.mark.gpu


def _ragged(lengths, lmax, d, dv, seed, sd=0.5):
    """q, k, v [groups][lmax][·] with the rows past each group's length zero."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = len(lengths)
    q = torch.randn(n, lmax, d, dtype=torch.float64, device="cuda", generator=g) * sd
    k = torch.randn(n, lmax, d, dtype=torch.float64, device="cuda", generator=g) * sd
    v = torch.randn(n, lmax, dv, dtype=torch.float64, device="cuda", generator=g)
    for w, t in enumerate(lengths):
        q[w, t:] = 0
        k[w, t:] = 0
        v[w, t:] = 0
    return q, k, v


def _same(got, want, precision, tol=1e-13):
    if precision == Precision.SPLIT:
        return torch.equal(got.nan_to_num(123.0), want.nan_to_num(123.0))
    if not torch.equal(torch.isnan(got), torch.isnan(want)):
        return False
    scale = max(want.nan_to_num().abs().max().item(), 1e-300)
    return (got.nan_to_num() - want.nan_to_num()).abs().max().item() <= tol * scale


CASES = {
    # group lengths, padded length, d, dv, conditions, scale
    "window_d128": ([700, 128, 1, 1500, 333, 64], 1500, 128, 64, A.window(100), 0.0884),
    "causal_d64": ([513, 40, 1024, 257], 1024, 64, 64, A.causal(), 1.0),
    "full_d32": ([90, 300, 7], 300, 32, 48, [], 1.0),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", [Precision.SPLIT, Precision.FP64])
def test_each_group_as_if_alone(name, precision):
    lengths, lmax, d, dv, cond, scale = CASES[name]
    q, k, v = _ragged(lengths, lmax, d, dv, seed=len(name))
    ql = torch.tensor(lengths, dtype=torch.int64)
    out, lse = A.attention_forward(q, k, v, cond, scale, precision, q_lengths=ql, k_lengths=ql)
    for w, t in enumerate(lengths):
        alone, lse_alone = A.attention_forward(q[w:w + 1, :t], k[w:w + 1, :t], v[w:w + 1, :t], cond, scale,
                                               precision)
        assert _same(out[w, :t], alone[0], precision), f"group {w}"
        assert _same(lse[w, :t], lse_alone[0], precision), f"group {w}: lse"
        assert torch.isnan(out[w, t:]).all(), f"group {w}: rows past the length written"
        want = _reference(q[w, :t], k[w, :t], v[w, :t], cond, scale)
        seen = ~torch.isnan(want)
        if seen.any():
            err = (out[w, :t][seen] - want[seen]).abs().max().item()
            assert err <= 1e-12 * want[seen].abs().max().item(), f"group {w}: {err}"


@pytest.mark.parametrize("precision", [Precision.SPLIT, Precision.FP64])
@pytest.mark.parametrize("shape", [
    ([200, 64, 333, 1], 333, 64, 64, A.causal(), 0.125),
    # d = 128 (the ragged bench batches' width): the backward takes the FP64 tiles in either form.
    ([150, 40, 260], 260, 128, 64, A.window(50), 0.0884),
])
def test_ragged_gradients(precision, shape):
    lengths, lmax, d, dv, cond, scale = shape
    q, k, v = _ragged(lengths, lmax, d, dv, seed=11)
    ql = torch.tensor(lengths, dtype=torch.int64)
    qa, ka, va = (t.clone().requires_grad_(True) for t in (q, k, v))
    out = A.attention(qa, ka, va, cond, scale, precision, q_lengths=ql, k_lengths=ql)
    g = torch.Generator(device="cuda").manual_seed(5)
    up = torch.randn(out.shape, dtype=torch.float64, device="cuda", generator=g)
    (out.nan_to_num() * up).sum().backward()
    for w, t in enumerate(lengths):
        qs, ks, vs = (x[w:w + 1, :t].clone().requires_grad_(True) for x in (q, k, v))
        alone = A.attention(qs, ks, vs, cond, scale, precision)
        (alone.nan_to_num() * up[w:w + 1, :t]).sum().backward()
        # The split backward (d <= 64) gives the same bits as alone; the FP64 one within rounding.
        form = precision if d <= 64 else Precision.FP64
        for name, a, b in (("q", qa.grad, qs.grad), ("k", ka.grad, ks.grad), ("v", va.grad, vs.grad)):
            assert _same(a[w, :t], b[0], form, tol=1e-12), f"d{name} of group {w}"
            assert (a[w, t:] == 0).all(), f"d{name} past the length of group {w}"


def test_lengths_outside_the_padding_are_refused():
    q, k, v = _ragged([5, 6], 6, 8, 8, seed=1)
    with pytest.raises(Exception, match="length"):
        A.attention_forward(q, k, v, q_lengths=torch.tensor([5, 7]), k_lengths=torch.tensor([5, 6]))


@pytest.mark.parametrize("precision", [Precision.SPLIT, Precision.FP64])
@pytest.mark.parametrize("lengths", [[0, 300, 0, 57], [0, 0]])
def test_empty_groups(precision, lengths):
    # A group of length 0 joins nothing: its rows are NaN and its gradients
    # zero, and the other groups come out as if alone; a batch of only
    # empty groups runs no tile at all.
    lmax, d, dv, cond, scale = 300, 32, 16, A.causal(), 0.5
    q, k, v = _ragged(lengths, lmax, d, dv, seed=13)
    ql = torch.tensor(lengths, dtype=torch.int64)
    qa, ka, va = (t.clone().requires_grad_(True) for t in (q, k, v))
    out = A.attention(qa, ka, va, cond, scale, precision, q_lengths=ql, k_lengths=ql)
    g = torch.Generator(device="cuda").manual_seed(6)
    up = torch.randn(out.shape, dtype=torch.float64, device="cuda", generator=g)
    (out.nan_to_num() * up).sum().backward()
    for w, t in enumerate(lengths):
        assert torch.isnan(out[w, t:]).all(), f"group {w}: rows past the length"
        for name, grad in (("q", qa.grad), ("k", ka.grad), ("v", va.grad)):
            assert (grad[w, t:] == 0).all(), f"d{name} past the length of group {w}"
        if t == 0:
            continue
        qs, ks, vs = (x[w:w + 1, :t].clone().requires_grad_(True) for x in (q, k, v))
        alone = A.attention(qs, ks, vs, cond, scale, precision)
        assert _same(out[w, :t], alone[0], precision), f"group {w}"
        (alone.nan_to_num() * up[w:w + 1, :t]).sum().backward()
        for name, a, b in (("q", qa.grad, qs.grad), ("k", ka.grad, ks.grad), ("v", va.grad, vs.grad)):
            assert _same(a[w, :t], b[0], precision, tol=1e-12), f"d{name} of group {w}"
