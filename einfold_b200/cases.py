"""Small runs of each product kernel, for a profiler (ncu) or a quick check.

    python -m einfold_b200.cases attention --groups 8 --t 2048 --d 64 [--backward]
    python -m einfold_b200.cases product --n 4096
    python -m einfold_b200.cases rank --n 67108864 [--repeat 3]
    python -m einfold_b200.cases ragged [--groups 64 --d 128 --window 512 --repeat 3]
    python -m einfold_b200.cases sparse

``attention`` runs the split causal attention forward (and backward) over
q, k, v normal(0, 1/8) and d_out normal(0, 1) (SplitMix64, seed 0);
``product`` runs einfold_split_gemm on two n x n uniform[-1, 1] FP64
matrices; ``rank`` ranks n uniform random 64-bit keys (each drawn from a
pool of n/2, so keys repeat) with einfold_rank_words and prints the keys
per second of the last of `repeat` runs, timed with CUDA events;
``ragged`` runs the split attention forward over ragged batches (lengths
log-uniform in [128, 8192], a window of |tq - tk| <= radius) and prints
the FLOP rate on the allowed pairs; ``sparse`` runs the discrimination
fold once on the sorting path's tables at 1/40 size (the bench's). Each
prints one line and exits 0 when the kernels ran.
"""
from __future__ import annotations

import argparse

import torch

from . import autograd as A
from . import synthetic as S
from .kernels import Precision


def attention(groups: int, t: int, d: int, backward: bool) -> None:
    n = groups * t * d
    q, k, v = (S.normal(0, salt, n, 1.0 / 8).view(groups, t, d) for salt in (3, 4, 5))
    out, lse = A.attention_forward(q, k, v, A.causal(), 1.0, Precision.SPLIT)
    if backward:
        d_out = S.normal(0, 6, n, 1.0).view(groups, t, d)
        A.attention_backward(q, k, v, out, lse, d_out, A.causal(), 1.0, Precision.SPLIT)
    torch.cuda.synchronize()
    print(f"attention groups={groups} t={t} d={d} backward={backward}: max|out| {out.abs().max().item():.6f}")


def product(n: int) -> None:
    a = S.uniform(0, 1, n * n).view(n, n)
    b = S.uniform(0, 2, n * n).view(n, n)
    c = A.matmul(a, b, Precision.SPLIT)
    torch.cuda.synchronize()
    print(f"product n={n}: max|C| {c.abs().max().item():.6f}")


def rank(n: int, repeat: int) -> None:
    import ctypes

    from . import _lib

    pool = S.u64(0, 7, max(n // 2, 1))
    pick = (S.u64(0, 8, n) % max(n // 2, 1)).to(torch.int64)
    words = pool[pick].contiguous()
    rank_ = torch.empty(n, dtype=torch.int32, device="cuda")
    first = torch.empty(n, dtype=torch.int32, device="cuda")
    k = ctypes.c_int64(0)
    lib = _lib.load()
    ms = 0.0
    for _ in range(max(repeat, 1)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        st = lib.einfold_rank_words(_lib.context(0), words.data_ptr(), n, rank_.data_ptr(), first.data_ptr(),
                                    ctypes.byref(k), None)
        e1.record()
        torch.cuda.synchronize()
        if st != _lib.OK:
            raise RuntimeError(lib.einfold_last_error().decode())
        ms = e0.elapsed_time(e1)
    print(f"rank n={n}: {k.value} distinct, {ms:.3f} ms, {n / ms / 1e6:.3f} Gkeys/s")


def ragged_lengths(groups: int, lo: int = 128, hi: int = 8192, seed: int = 0) -> torch.Tensor:
    """Group lengths log-uniform in [lo, hi] (SplitMix64 units, salt 9)."""
    u = S.units(seed, 9, groups, device="cpu").to(torch.float64)
    return torch.exp(torch.log(torch.tensor(float(lo))) + u * (torch.log(torch.tensor(float(hi))) -
                                                             torch.log(torch.tensor(float(lo))))).floor().to(torch.int64)


def ragged_inputs(groups: int, d: int, seed: int = 0):
    """q, k, v [groups][8192][d], normal(0, 1/sqrt(d)), zero past each group's length."""
    lengths = ragged_lengths(groups, seed=seed)
    lmax = int(lengths.max())
    n = groups * lmax * d
    q, k, v = (S.normal(seed, salt, n, d ** -0.5).view(groups, lmax, d) for salt in (3, 4, 5))
    pos = torch.arange(lmax, device=q.device)[None, :, None]
    pad = pos >= lengths.to(q.device)[:, None, None]
    for x in (q, k, v):
        x.masked_fill_(pad, 0.0)
    return q, k, v, lengths


def allowed_pairs(lengths: torch.Tensor, radius: int) -> int:
    """Pairs with |tq - tk| <= radius inside each group."""
    total = 0
    for t in lengths.tolist():
        x = torch.arange(t, dtype=torch.int64)
        total += int((torch.clamp(x + radius, max=t - 1) - torch.clamp(x - radius, min=0) + 1).sum())
    return total


def ragged(groups: int, d: int, radius: int, repeat: int) -> None:
    q, k, v, lengths = ragged_inputs(groups, d)
    flop = 4.0 * d * allowed_pairs(lengths, radius)
    ms = 0.0
    for _ in range(max(repeat, 1)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        A.attention_forward(q, k, v, A.window(radius), d ** -0.5, Precision.SPLIT, q_lengths=lengths,
                            k_lengths=lengths)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    from .kernels import last_call

    print(f"ragged groups={groups} d={d} window={radius} rows={int(lengths.sum())}: {ms:.3f} ms, "
          f"{flop / ms / 1e9:.2f} TFLOP/s (attention kernel {last_call.product_ms:.3f} ms)")


def sparse() -> None:
    import os
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    from . import kernels as K

    a, b, pairs = bench._sparse_tables()
    got = K.fold(bench._matmul_fold(), K.Relation(a.schema, [a]), K.Relation(b.schema, [b]),
                 options=K.Options(result_on_device=True))
    rows = sum(batch.rows for batch in got.batches)
    for batch in got.batches:
        batch.release()
    print(f"sparse: {pairs} pair products, {rows} groups ({got.algorithm.name.lower()})")


def main() -> None:
    p = argparse.ArgumentParser()
    sub = p.add_subparsers(dest="case", required=True)
    pa = sub.add_parser("attention")
    pa.add_argument("--groups", type=int, default=8)
    pa.add_argument("--t", type=int, default=2048)
    pa.add_argument("--d", type=int, default=64)
    pa.add_argument("--backward", action="store_true")
    pp = sub.add_parser("product")
    pp.add_argument("--n", type=int, default=4096)
    pg = sub.add_parser("ragged")
    pg.add_argument("--groups", type=int, default=64)
    pg.add_argument("--d", type=int, default=128)
    pg.add_argument("--window", type=int, default=512)
    pg.add_argument("--repeat", type=int, default=3)
    sub.add_parser("sparse")
    pr = sub.add_parser("rank")
    pr.add_argument("--n", type=int, default=1 << 26)
    pr.add_argument("--repeat", type=int, default=3)
    args = p.parse_args()
    if args.case == "attention":
        attention(args.groups, args.t, args.d, args.backward)
    elif args.case == "rank":
        rank(args.n, args.repeat)
    elif args.case == "ragged":
        ragged(args.groups, args.d, args.window, args.repeat)
    elif args.case == "sparse":
        sparse()
    else:
        product(args.n)


if __name__ == "__main__":
    main()
