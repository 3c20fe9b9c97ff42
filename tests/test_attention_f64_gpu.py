"""The FP64 form of the attention forward on the FP64 tensor pipe (mma.sync
f64) against torch float64 on the same operands: odd and even feature and
value widths (the cp.async and the element-by-element tile loads), masks,
scales, ragged groups, and rows that join no key; and the same guard
declines as the split form's."""
import ctypes

import numpy as np
import pytest
import torch

from einfold_b200 import _lib
from einfold_b200 import autograd as A
from einfold_b200.ir import Comparison
from einfold_b200.kernels import Precision

pytestmark = pytest.mark.gpu

GE, LE, LT = Comparison.GREATER_OR_EQUAL, Comparison.LESS_OR_EQUAL, Comparison.LESS


def _reference(q, k, v, conditions, scale, q_len=None, k_len=None):
    lq, lk = q.shape[-2], k.shape[-2]
    x = torch.arange(lq, device=q.device)[:, None]
    j = torch.arange(lk, device=q.device)[None, :]
    allowed = torch.ones(q.shape[0], lq, lk, dtype=torch.bool, device=q.device)
    for cmp, off in conditions:
        rhs = j + off
        allowed &= {Comparison.LESS: x < rhs, Comparison.LESS_OR_EQUAL: x <= rhs, Comparison.GREATER: x > rhs,
                    Comparison.GREATER_OR_EQUAL: x >= rhs}[Comparison(cmp)]
    if q_len is not None:
        allowed &= (x[None] < q_len[:, None, None]) & (j[None] < k_len[:, None, None])
    s = (q @ k.transpose(-1, -2)) * scale
    s = s.masked_fill(~allowed, float("-inf"))
    some = allowed.any(-1, keepdim=True)
    out = torch.softmax(torch.where(some, s, torch.zeros_like(s)), dim=-1) @ v
    return out, some


CASES = {
    "causal_d64": (3, 300, 300, 64, 64, A.causal(), 1.0),
    "odd_widths": (2, 77, 150, 3, 5, [], 0.5),
    "wide": (2, 130, 200, 128, 130, A.window(17), 0.125),
    "d100": (2, 64, 64, 100, 33, [(GE, 5)], 1.0),  # the first 5 queries join nothing
    "one_feature": (4, 40, 90, 1, 1, [(LT, 30)], 2.0),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_tensor_pipe_forward_matches_torch(name):
    w, lq, lk, d, dv, cond, scale = CASES[name]
    g = torch.Generator(device="cuda").manual_seed(len(name))
    q = torch.randn(w, lq, d, dtype=torch.float64, device="cuda", generator=g) * 0.4
    k = torch.randn(w, lk, d, dtype=torch.float64, device="cuda", generator=g) * 0.4
    v = torch.randn(w, lk, dv, dtype=torch.float64, device="cuda", generator=g)
    out, lse = A.attention_forward(q, k, v, cond, scale, Precision.FP64)
    want, some = _reference(q, k, v, cond, scale)
    rows = some.expand_as(want)
    err = (out[rows] - want[rows]).abs().max().item()
    assert err <= 1e-12 * v.abs().max().item(), err
    # lse = m + ln z on the rows that join a key.
    s = (q @ k.transpose(-1, -2)) * scale
    x = torch.arange(lq, device="cuda")[:, None]
    j = torch.arange(lk, device="cuda")[None, :]
    allowed = torch.ones(lq, lk, dtype=torch.bool, device="cuda")
    for cmp, off in cond:
        rhs = j + off
        allowed &= {Comparison.LESS: x < rhs, Comparison.LESS_OR_EQUAL: x <= rhs, Comparison.GREATER: x > rhs,
                    Comparison.GREATER_OR_EQUAL: x >= rhs}[Comparison(cmp)]
    want_lse = torch.logsumexp(s.masked_fill(~allowed, float("-inf")), -1)
    r = some[..., 0]
    assert (lse[r] - want_lse[r]).abs().max().item() <= 1e-12 * want_lse[r].abs().max().item() + 1e-13


def test_fp64_tensor_pipe_forward_on_ragged_groups():
    w, lmax, d, dv = 5, 200, 64, 48
    g = torch.Generator(device="cuda").manual_seed(3)
    q = torch.randn(w, lmax, d, dtype=torch.float64, device="cuda", generator=g) * 0.3
    k = torch.randn(w, lmax, d, dtype=torch.float64, device="cuda", generator=g) * 0.3
    v = torch.randn(w, lmax, dv, dtype=torch.float64, device="cuda", generator=g)
    lengths = torch.tensor([200, 1, 64, 65, 130], dtype=torch.int64, device="cuda")
    out, _ = A.attention_forward(q, k, v, A.window(20), 1.0, Precision.FP64, q_lengths=lengths, k_lengths=lengths)
    want, some = _reference(q, k, v, A.window(20), 1.0, lengths, lengths)
    rows = some.expand_as(want)
    assert (out[rows] - want[rows]).abs().max().item() <= 1e-12 * v.abs().max().item()


def test_fp64_and_split_forms_agree_and_both_guard_an_underflow():
    # Within their tolerances on ordinary values.
    g = torch.Generator(device="cuda").manual_seed(5)
    q, k = (torch.randn(2, 256, 64, dtype=torch.float64, device="cuda", generator=g) * 0.125 for _ in range(2))
    v = torch.randn(2, 256, 64, dtype=torch.float64, device="cuda", generator=g)
    o64, _ = A.attention_forward(q, k, v, A.causal(), 1.0, Precision.FP64)
    osp, _ = A.attention_forward(q, k, v, A.causal(), 1.0, Precision.SPLIT)
    assert (o64 - osp).abs().max().item() <= 2e-12 * v.abs().max().item()
    # Subnormal values: a term that underflows could lose more than rounding
    # of the result, so the guard (Bounds::hold, fused.rs:1058-1086)
    # declines, in both forms.
    lib = _lib.load()
    qs = torch.randn(1, 64, 8, dtype=torch.float64, device="cuda", generator=g) * 0.1
    ks = torch.randn(1, 64, 8, dtype=torch.float64, device="cuda", generator=g) * 0.1
    vs = torch.full((1, 64, 8), 1e-310, dtype=torch.float64, device="cuda")
    out = torch.empty(1, 64, 8, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for precision in (0, 1):
        st = lib.einfold_attention_forward(_lib.context(0), qs.data_ptr(), ks.data_ptr(), vs.data_ptr(),
                                           out.data_ptr(), None, 1, 64, 64, 8, 8, 0, None, None, 1.0, precision, 0,
                                           ctypes.c_void_p(1), None)  # stream 1: cudaStreamLegacy
        assert st == _lib.DECLINED


@pytest.mark.parametrize("shape", [(2, 200, 64, 64, "causal"), (3, 77, 3, 5, "window"), (2, 130, 64, 40, "ragged")])
def test_fp64_tensor_pipe_backward_matches_torch(shape):
    # The FP64 backward (keys-as-rows and queries-as-rows kernels on the FP64
    # tensor pipe) against torch float64 autograd of the same attention.
    w, l, d, dv, kind = shape
    g = torch.Generator(device="cuda").manual_seed(l)
    q = torch.randn(w, l, d, dtype=torch.float64, device="cuda", generator=g) * 0.3
    k = torch.randn(w, l, d, dtype=torch.float64, device="cuda", generator=g) * 0.3
    v = torch.randn(w, l, dv, dtype=torch.float64, device="cuda", generator=g)
    d_out = torch.randn(w, l, dv, dtype=torch.float64, device="cuda", generator=g)
    cond = A.causal() if kind == "causal" else A.window(9)
    lengths = torch.tensor([l, 57][:w], dtype=torch.int64, device="cuda") if kind == "ragged" else None
    if lengths is not None:
        pos = torch.arange(l, device="cuda")[None, :, None] < lengths[:, None, None]
        q, k, v, d_out = q * pos, k * pos, v * pos, d_out * pos
    out, lse = A.attention_forward(q, k, v, cond, 1.0, Precision.FP64, q_lengths=lengths, k_lengths=lengths)
    dq, dk, dvv = A.attention_backward(q, k, v, out, lse, d_out, cond, 1.0, Precision.FP64, q_lengths=lengths,
                                       k_lengths=lengths)
    qr, kr, vr = (t.clone().requires_grad_(True) for t in (q, k, v))
    want, some = _reference(qr, kr, vr, cond, 1.0, lengths, lengths)
    gq, gk, gv = torch.autograd.grad(want, (qr, kr, vr), d_out * some)
    for got, ref in ((dq, gq), (dk, gk), (dvv, gv)):
        assert (got - ref).abs().max().item() <= 1e-11 * max(ref.abs().max().item(), 1e-300)
