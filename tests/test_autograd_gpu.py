"""Attention and matrix-product folds over torch tensors: forward against a
torch float64 restatement of the same softmax average, backward against
torch's autograd of it and against central finite differences (eps = 1e-6)
on 32 sampled entries, in both the split and the FP64 form."""
import numpy as np
import pytest
import torch

from einfold_b200 import autograd as A
from einfold_b200.ir import Comparison
from einfold_b200.kernels import Precision

pytestmark = pytest.mark.gpu

GE = Comparison.GREATER_OR_EQUAL


def _reference(q, k, v, conditions, scale):
    """softmax(scale·q·kᵀ) · v over the allowed pairs, in torch float64."""
    lq, lk = q.shape[-2], k.shape[-2]
    x = torch.arange(lq, device=q.device)[:, None]
    j = torch.arange(lk, device=q.device)[None, :]
    allowed = torch.ones(lq, lk, dtype=torch.bool, device=q.device)
    for cmp, off in conditions:
        rhs = j + off
        allowed &= {Comparison.LESS: x < rhs, Comparison.LESS_OR_EQUAL: x <= rhs, Comparison.GREATER: x > rhs,
                    Comparison.GREATER_OR_EQUAL: x >= rhs}[Comparison(cmp)]
    s = scale * (q @ k.transpose(-1, -2))
    s = s.masked_fill(~allowed, float("-inf"))
    # A query with no allowed key has no row (NaN here), and no gradient.
    some = allowed.any(-1)[:, None]
    out = torch.softmax(torch.where(some, s, torch.zeros_like(s)), dim=-1) @ v
    return torch.where(some, out, torch.full_like(out, float("nan")))


def _inputs(shape_q, shape_k, dv, seed, sd=0.5):
    g = torch.Generator(device="cuda").manual_seed(seed)
    q = torch.randn(*shape_q, dtype=torch.float64, device="cuda", generator=g) * sd
    k = torch.randn(*shape_k, dtype=torch.float64, device="cuda", generator=g) * sd
    v = torch.randn(*shape_k[:-1], dv, dtype=torch.float64, device="cuda", generator=g)
    return q, k, v


SHAPES = {
    "causal": ((2, 3, 256, 64), (2, 3, 256, 64), 64, A.causal(), 1.0),
    "window_scaled": ((4, 200, 32), (4, 200, 32), 48, A.window(40), 0.125),
    "cross": ((3, 130, 16), (3, 300, 16), 8, [], 1.0),
    "late_start": ((2, 150, 64), (2, 150, 64), 64, [(GE, 20)], 1.0),  # the first 20 queries see no key
}


@pytest.mark.parametrize("name", list(SHAPES))
@pytest.mark.parametrize("precision", [Precision.SPLIT, Precision.FP64])
def test_forward_and_gradients_match_torch_float64(name, precision):
    sq, sk, dv, cond, scale = SHAPES[name]
    q, k, v = _inputs(sq, sk, dv, seed=len(name))
    qr, kr, vr = (t.clone().requires_grad_(True) for t in (q, k, v))
    want = _reference(qr, kr, vr, cond, scale)
    qa, ka, va = (t.clone().requires_grad_(True) for t in (q, k, v))
    got = A.attention(qa, ka, va, cond, scale, precision)
    seen = ~torch.isnan(want)
    assert torch.equal(seen, ~torch.isnan(got)), "rows without keys differ"
    err = (got[seen] - want[seen]).abs().max().item()
    assert err <= 1e-12 * want[seen].abs().max().item(), err
    g = torch.randn_like(want)
    (want.nan_to_num() * g).sum().backward()
    (got.nan_to_num() * g).sum().backward()
    for which, a, b in (("q", qa.grad, qr.grad), ("k", ka.grad, kr.grad), ("v", va.grad, vr.grad)):
        scale_ = b.abs().max().item()
        e = (a - b).abs().max().item()
        assert e <= 1e-11 * max(scale_, 1e-300), f"d{which}: {e / scale_:.3e}"


@pytest.mark.parametrize("precision", [Precision.SPLIT, Precision.FP64])
def test_gradients_against_finite_differences(precision):
    q, k, v = _inputs((2, 96, 32), (2, 96, 32), 32, seed=11)
    cond = A.causal()
    g = torch.randn(2, 96, 32, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))

    def loss(q_, k_, v_):
        out, _ = A.attention_forward(q_, k_, v_, cond, 1.0, Precision.FP64)
        return (out * g).sum().item()

    qa, ka, va = (t.clone().requires_grad_(True) for t in (q, k, v))
    (A.attention(qa, ka, va, cond, 1.0, precision) * g).sum().backward()
    rng = np.random.default_rng(5)
    eps = 1e-6
    # 11 entries of each of q, k and v: 33 in all.
    for which, t, grad in (("q", q, qa.grad), ("k", k, ka.grad), ("v", v, va.grad)):
        for idx in rng.choice(t.numel(), 11, replace=False):
            plus, minus = t.clone(), t.clone()
            plus.view(-1)[idx] += eps
            minus.view(-1)[idx] -= eps
            args_p = [plus if w == which else x for w, x in (("q", q), ("k", k), ("v", v))]
            args_m = [minus if w == which else x for w, x in (("q", q), ("k", k), ("v", v))]
            fd = (loss(*args_p) - loss(*args_m)) / (2 * eps)
            an = grad.reshape(-1)[idx].item()
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (which, int(idx), fd, an)


@pytest.mark.parametrize("precision", [Precision.SPLIT, Precision.FP64])
def test_matmul_fold_gradients(precision):
    gen = torch.Generator(device="cuda").manual_seed(9)
    a = torch.rand(300, 200, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
    b = torch.rand(200, 150, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
    dc = torch.randn(300, 150, dtype=torch.float64, device="cuda", generator=gen)
    aa, bb = a.clone().requires_grad_(True), b.clone().requires_grad_(True)
    c = A.matmul(aa, bb, precision)
    want = a @ b
    assert (c - want).abs().max().item() <= 1e-12 * want.abs().max().item()
    (c * dc).sum().backward()
    for got, want in ((aa.grad, dc @ b.T), (bb.grad, a.T @ dc)):
        assert (got - want).abs().max().item() <= 1e-12 * want.abs().max().item()
    # Finite differences on 32 entries of each input (the product is linear
    # in each, so the central difference is exact up to rounding).
    rng = np.random.default_rng(1)
    eps = 1e-6
    for t, grad, is_a in ((a, aa.grad, True), (b, bb.grad, False)):
        for idx in rng.choice(t.numel(), 32, replace=False):
            p, m = t.clone(), t.clone()
            p.view(-1)[idx] += eps
            m.view(-1)[idx] -= eps
            lp = ((p @ b if is_a else a @ p) * dc).sum().item()
            lm = ((m @ b if is_a else a @ m) * dc).sum().item()
            assert abs((lp - lm) / (2 * eps) - grad.view(-1)[idx].item()) <= 1e-6
