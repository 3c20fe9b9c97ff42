"""Differentiable folds over torch tensors on the GPU, through the C ABI.

``attention`` is the pipeline of ``einfold_kernels::pipeline`` for product
scores, a softmax shifted by the kept maximum and an average normalised by
the kept groups (fused.rs:694-1019), over FP64 tensors [..., l, d]; its
backward recomputes the scores tile by tile from the saved log-sum-exp.
``matmul`` is the dense positional fold SUM(a.v * b.v) GROUP BY i, k
(dense.rs) over FP64 matrices; its gradients are the folds a gradient SQL
program writes, dA = dC·Bᵀ and dB = Aᵀ·dC. Both run the split form (int8
digit products on the tensor cores, FP64 combine) unless
``precision=Precision.FP64``.

The reference's Python extension differentiates folds by writing gradient
SQL; these functions are the tensor-level counterparts for training loops.
"""
from __future__ import annotations

import ctypes
from typing import Sequence, Tuple

import torch

from . import _lib
from .ir import Comparison
from .kernels import Precision, _raise

__all__ = ["attention", "attention_forward", "attention_backward", "matmul", "Conditions", "causal", "window",
           "Declined"]


class Declined(RuntimeError):
    """The reference's pipeline would return None here (its overflow or
    underflow guards fired): the caller runs its host plan instead."""


Conditions = Sequence[Tuple[Comparison, int]]


def causal() -> Conditions:
    """q.t >= k.t: each query sees the keys at or before it."""
    return [(Comparison.GREATER_OR_EQUAL, 0)]


def window(radius: int) -> Conditions:
    """|q.t - k.t| <= radius."""
    return [(Comparison.LESS_OR_EQUAL, radius), (Comparison.GREATER_OR_EQUAL, -radius)]


def _check(t: torch.Tensor, name: str) -> torch.Tensor:
    if not t.is_cuda or t.dtype != torch.float64:
        raise TypeError(f"{name} must be a float64 CUDA tensor")
    return t.contiguous()


def _conditions(conditions: Conditions):
    n = len(conditions)
    cmp = (ctypes.c_int32 * max(n, 1))(*[int(c) for c, _ in conditions])
    off = (ctypes.c_int64 * max(n, 1))(*[int(o) for _, o in conditions])
    return n, cmp, off


def _stream(device: int) -> int:
    """torch's current stream on `device` as the library's stream argument.
    The legacy default stream (handle 0) goes as cudaStreamLegacy (1): a
    null stream would mean the context's own stream, which does not wait
    for work queued on the default one (the operands' copies, say)."""
    return torch.cuda.current_stream(device).cuda_stream or 1


def _call(fn, device: int, *args) -> _lib.Result:
    info = _lib.Result()
    stream = _stream(device)
    st = fn(_lib.context(device), *args, ctypes.c_void_p(stream), ctypes.byref(info))
    if st == _lib.DECLINED:
        raise Declined(info.message.decode(errors="replace"))
    from .kernels import last_call

    last_call.kernels_launched = info.kernels_launched
    last_call.device_ms = info.device_ms
    last_call.product_ms = info.product_ms
    last_call.product_ops = info.product_ops
    last_call.schedule = info.schedule
    last_call.graph = info.graph
    last_call.message = info.message.decode(errors="replace")
    if st != _lib.OK:
        _raise(st, info.message.decode(errors="replace"))
    return info


def _batches(lead) -> int:
    n = 1
    for x in lead:
        n *= x
    return n


def _lengths(x, lead, name, device):
    """A ragged batch's lengths as a contiguous int64 tensor, one value per
    batch, on the operands' device; or None."""
    if x is None:
        return None
    x = torch.as_tensor(x, dtype=torch.int64)
    if x.numel() != _batches(lead):
        raise ValueError(f"{name} needs one length per batch ({_batches(lead)}), not {x.numel()}")
    return x.reshape(-1).to(device).contiguous()


def _ptr(x):
    return x.data_ptr() if x is not None else None


def attention_forward(q: torch.Tensor, k: torch.Tensor, v: torch.Tensor, conditions: Conditions = (),
                      scale: float = 1.0, precision: Precision = Precision.SPLIT, slices: int = 0,
                      q_lengths=None, k_lengths=None) -> Tuple[torch.Tensor, torch.Tensor]:
    """out [..., lq, dv] and lse [..., lq] of softmax(scale·q·kᵀ) · v over the
    allowed pairs (q.t <cmp> k.t + off for every condition). Rows with no
    allowed key are NaN. Raises ``Declined`` where the reference's overflow
    or underflow guards send the pipeline back to the host plan.

    Ragged batches: ``q_lengths`` / ``k_lengths`` (one per batch) say how
    many of the padded rows of q, and of k and v, each batch uses; queries
    past their length are NaN rows, keys past it are never joined. The
    padding rows must hold finite values (zeros, say)."""
    q, k, v = _check(q, "q"), _check(k, "k"), _check(v, "v")
    *lead, lq, d = q.shape
    lk, dv = k.shape[-2], v.shape[-1]
    if tuple(k.shape[:-2]) != tuple(lead) or tuple(v.shape[:-2]) != tuple(lead) or k.shape[-1] != d or \
            v.shape[-2] != lk:
        raise ValueError("q [..., lq, d], k [..., lk, d] and v [..., lk, dv] must agree")
    out = torch.full((*lead, lq, dv), float("nan"), dtype=torch.float64, device=q.device)
    lse = torch.full((*lead, lq), float("nan"), dtype=torch.float64, device=q.device)
    n, cmp, off = _conditions(conditions)
    ql = _lengths(q_lengths, lead, "q_lengths", q.device)
    kl = _lengths(k_lengths, lead, "k_lengths", q.device)
    lib = _lib.load()
    if ql is None and kl is None:
        _call(lib.einfold_attention_forward, q.device.index or 0, q.data_ptr(), k.data_ptr(), v.data_ptr(),
              out.data_ptr(), lse.data_ptr(), _batches(lead), lq, lk, d, dv, n, cmp, off, float(scale),
              Precision(precision).value, int(slices))
    else:
        _call(lib.einfold_attention_forward_ragged, q.device.index or 0, q.data_ptr(), k.data_ptr(), v.data_ptr(),
              out.data_ptr(), lse.data_ptr(), _batches(lead), lq, lk, d, dv, _ptr(ql), _ptr(kl), n, cmp, off,
              float(scale), Precision(precision).value, int(slices))
    return out, lse


def attention_backward(q, k, v, out, lse, d_out, conditions: Conditions = (), scale: float = 1.0,
                       precision: Precision = Precision.SPLIT, q_lengths=None,
                       k_lengths=None) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """d_q, d_k, d_v of ``attention_forward``'s out for the upstream d_out
    (ragged batches as there: the padding rows' gradients are zero, and
    d_out's padding rows must be finite)."""
    q, k, v = _check(q, "q"), _check(k, "k"), _check(v, "v")
    out, lse, d_out = _check(out, "out"), _check(lse, "lse"), _check(d_out, "d_out")
    *lead, lq, d = q.shape
    lk, dv = k.shape[-2], v.shape[-1]
    d_q, d_k, d_v = torch.empty_like(q), torch.empty_like(k), torch.empty_like(v)
    n, cmp, off = _conditions(conditions)
    ql = _lengths(q_lengths, lead, "q_lengths", q.device)
    kl = _lengths(k_lengths, lead, "k_lengths", q.device)
    lib = _lib.load()
    if ql is None and kl is None:
        _call(lib.einfold_attention_backward, q.device.index or 0, q.data_ptr(), k.data_ptr(), v.data_ptr(),
              out.data_ptr(), lse.data_ptr(), d_out.data_ptr(), d_q.data_ptr(), d_k.data_ptr(), d_v.data_ptr(),
              _batches(lead), lq, lk, d, dv, n, cmp, off, float(scale), Precision(precision).value)
    else:
        _call(lib.einfold_attention_backward_ragged, q.device.index or 0, q.data_ptr(), k.data_ptr(), v.data_ptr(),
              out.data_ptr(), lse.data_ptr(), d_out.data_ptr(), d_q.data_ptr(), d_k.data_ptr(), d_v.data_ptr(),
              _batches(lead), lq, lk, d, dv, _ptr(ql), _ptr(kl), n, cmp, off, float(scale),
              Precision(precision).value)
    return d_q, d_k, d_v


class _Attention(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, k, v, conditions, scale, precision, slices, q_lengths, k_lengths):
        out, lse = attention_forward(q, k, v, conditions, scale, precision, slices, q_lengths, k_lengths)
        ctx.save_for_backward(q, k, v, out, lse)
        ctx.conditions, ctx.scale, ctx.precision = conditions, scale, precision
        ctx.lengths = (q_lengths, k_lengths)
        return out

    @staticmethod
    def backward(ctx, d_out):
        q, k, v, out, lse = ctx.saved_tensors
        d_out = d_out.contiguous()
        if ctx.lengths != (None, None):
            # The padding rows carry no gradient (and must be finite).
            d_out = torch.nan_to_num(d_out, nan=0.0)
        d_q, d_k, d_v = attention_backward(q, k, v, out, lse, d_out, ctx.conditions, ctx.scale, ctx.precision,
                                           *ctx.lengths)
        return d_q, d_k, d_v, None, None, None, None, None, None


def attention(q: torch.Tensor, k: torch.Tensor, v: torch.Tensor, conditions: Conditions = (), scale: float = 1.0,
              precision: Precision = Precision.SPLIT, slices: int = 0, q_lengths=None,
              k_lengths=None) -> torch.Tensor:
    """Differentiable softmax attention (see ``attention_forward``; ragged
    batches by ``q_lengths`` / ``k_lengths``)."""
    return _Attention.apply(q, k, v, list(conditions), float(scale), Precision(precision), int(slices), q_lengths,
                            k_lengths)


def _gemm(a: torch.Tensor, b: torch.Tensor, b_transposed: bool, precision: Precision, slices: int) -> torch.Tensor:
    """C = A·B for [..., m, k] A and B [..., k, n] (or [..., n, k] transposed)."""
    a, b = _check(a, "a"), _check(b, "b")
    *lead, m, kk = a.shape
    n = b.shape[-2] if b_transposed else b.shape[-1]
    c = torch.empty((*lead, m, n), dtype=torch.float64, device=a.device)
    lib = _lib.load()
    device = a.device.index or 0
    stream = ctypes.c_void_p(_stream(device))
    if Precision(precision) == Precision.SPLIT:
        st = lib.einfold_split_gemm(_lib.context(device), a.data_ptr(), b.data_ptr(), c.data_ptr(), _batches(lead), m,
                                    n, kk, int(b_transposed), int(slices), stream)
    else:
        st = lib.einfold_fp64_gemm(_lib.context(device), a.data_ptr(), b.data_ptr(), c.data_ptr(), _batches(lead), m,
                                   n, kk, int(b_transposed), stream)
    if st != _lib.OK:
        _raise(st, lib.einfold_last_error().decode(errors="replace"))
    return c


class _MatMul(torch.autograd.Function):
    @staticmethod
    def forward(ctx, a, b, precision, slices):
        ctx.save_for_backward(a, b)
        ctx.precision, ctx.slices = precision, slices
        return _gemm(a, b, False, precision, slices)

    @staticmethod
    def backward(ctx, d_c):
        a, b = ctx.saved_tensors
        d_c = d_c.contiguous()
        # dA = dC·Bᵀ: B [k][n] is Bᵀ's transposed layout. dB = Aᵀ·dC.
        d_a = _gemm(d_c, b, True, ctx.precision, ctx.slices) if ctx.needs_input_grad[0] else None
        d_b = _gemm(a.transpose(-1, -2).contiguous(), d_c, False, ctx.precision, ctx.slices) \
            if ctx.needs_input_grad[1] else None
        return d_a, d_b, None, None


def matmul(a: torch.Tensor, b: torch.Tensor, precision: Precision = Precision.SPLIT, slices: int = 0) -> torch.Tensor:
    """Differentiable A·B of FP64 [..., m, k] and [..., k, n] tensors: the
    matrix-product fold; the split form needs every value finite."""
    return _MatMul.apply(a, b, Precision(precision), int(slices))
