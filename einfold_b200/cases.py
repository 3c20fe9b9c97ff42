"""Small runs of each product kernel, for a profiler (ncu) or a quick check.

    python -m einfold_b200.cases attention --groups 8 --t 2048 --d 64 [--backward]
    python -m einfold_b200.cases product --n 4096

``attention`` runs the split causal attention forward (and backward) over
q, k, v normal(0, 1/8) and d_out normal(0, 1) (SplitMix64, seed 0);
``product`` runs einfold_split_gemm on two n x n uniform[-1, 1] FP64
matrices. Each prints one line and exits 0 when the kernels ran.
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
    args = p.parse_args()
    if args.case == "attention":
        attention(args.groups, args.t, args.d, args.backward)
    else:
        product(args.n)


if __name__ == "__main__":
    main()
