"""Small runs of each product kernel, for a profiler (ncu) or a quick check.

    python -m einfold_b200.cases attention --groups 8 --t 2048 --d 64 [--backward]
    python -m einfold_b200.cases product --n 4096
    python -m einfold_b200.cases rank --n 67108864 [--repeat 3]
    python -m einfold_b200.cases ragged [--groups 64 --d 128 --window 512 --repeat 3]
    python -m einfold_b200.cases sparse
    python -m einfold_b200.cases smoother [--groups 64 --x 1048576 --y 256]

``attention`` runs the split causal attention forward (and backward) over
q, k, v normal(0, 1/8) and d_out normal(0, 1) (SplitMix64, seed 0);
``product`` runs einfold_split_gemm on two n x n uniform[-1, 1] FP64
matrices; ``rank`` ranks n uniform random 64-bit keys (each drawn from a
pool of n/2, so keys repeat) with einfold_rank_words and prints the keys
per second of the last of `repeat` runs, timed with CUDA events;
``ragged`` runs the split attention forward over ragged batches (lengths
log-uniform in [128, 8192], a window of |tq - tk| <= radius) and prints
the FLOP rate on the allowed pairs; ``sparse`` runs the discrimination
fold once on the sorting path's tables at 1/40 size (the bench's);
``smoother`` runs the Gaussian smoother pipeline (x positions a group, y
key positions, h = 0.01) once. Each prints one line and exits 0 when the
kernels ran.
"""
from __future__ import annotations

import argparse

import torch

from . import autograd as A
from . import synthetic as S
from .kernels import Precision


def attention(groups: int, t: int, d: int, backward: bool, precision: Precision = Precision.SPLIT) -> None:
    n = groups * t * d
    q, k, v = (S.normal(0, salt, n, 1.0 / 8).view(groups, t, d) for salt in (3, 4, 5))
    out, lse = A.attention_forward(q, k, v, A.causal(), 1.0, precision)
    if backward:
        d_out = S.normal(0, 6, n, 1.0).view(groups, t, d)
        A.attention_backward(q, k, v, out, lse, d_out, A.causal(), 1.0, precision)
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
    from . import ir
    from . import kernels as K

    a, b = S.sorting_tables(50_000)
    pairs = S.joined_pairs(a.column(1).to_numpy(), b.column(0).to_numpy())
    e = ir.EQ
    f = ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                [ir.Output(0), ir.Output(2)])
    got = K.fold(f, K.Relation(a.schema, [a]), K.Relation(b.schema, [b]), options=K.Options(result_on_device=True))
    rows = sum(batch.rows for batch in got.batches)
    for batch in got.batches:
        batch.release()
    print(f"sparse: {pairs} pair products, {rows} groups ({got.algorithm.name.lower()})")


def small_fold_tables(nulls: bool, seed: int = 0):
    """The plain matmul fold's tables at 512 x 512 . 512 x 256: a(i, j, v)
    with every (i, j) of 512 x 512 and b(j, k, v) with every (j, k) of
    512 x 256, v uniform[-1, 1] (SplitMix64 salts 31, 32), with `nulls` 1%
    of b's v NULL (independent draws, salt 33); rows shuffled (salts 34, 35)
    and cut into four batches at random rows (salts 36, 37). Host Arrow
    (schema, batches) pairs."""
    import numpy as np
    import pyarrow as pa

    def table(names, extents, salt_v, salt_perm, salt_cut, null_salt=None):
        n = int(np.prod(extents))
        keys = np.indices(extents).reshape(len(extents), -1)
        vals = S.uniform(seed, salt_v, n, device="cpu").numpy()
        mask = S.units(seed, null_salt, n, device="cpu").numpy() < 0.01 if null_salt else None
        order = np.argsort(S.u64(seed, salt_perm, n, device="cpu").numpy(), kind="stable")
        cuts = np.sort((S.units(seed, salt_cut, 3, device="cpu").numpy() * n).astype(np.int64))
        bounds = [0, *cuts.tolist(), n]
        schema = pa.schema([(c, pa.int64()) for c in names] + [("v", pa.float64())])
        batches = []
        for lo, hi in zip(bounds[:-1], bounds[1:]):
            rows = order[lo:hi]
            cols = [pa.array(keys[c][rows]) for c in range(len(names))]
            cols.append(pa.array(vals[rows], mask=mask[rows] if mask is not None else None))
            batches.append(pa.record_batch(cols, schema=schema))
        return schema, batches

    a = table(["i", "j"], [512, 512], 31, 34, 36)
    b = table(["j", "k"], [512, 256], 32, 35, 37, 33 if nulls else None)
    return a, b


def smoother_pipeline(h: float = 0.01):
    """The Gaussian smoother as a pipeline over q(b, t, d, x), k(b, t, d, x)
    and v(b, t, x): scores the row expression -power(q.x - k.x, 2) over one
    feature d, FP64 weights exp(s / h) without a shift, normalised by the
    kept groups, so out(b, t) = sum_y w v / sum_y w with
    w = exp(-power(x - y, 2) / h)."""
    from . import ir

    E = ir.Dimension(ir.KeyEquality.EQUAL)
    I, D, J, B = 0, 1, 2, 3
    diff = ir.Expression.column(0, 3).binary(ir.Binary.SUBTRACT, ir.Expression.column(1, 3))
    scores = diff.binary(ir.Binary.POWER, ir.Expression.literal(2.0)).unary(ir.Unary.NEGATE)
    producer = ir.Fold([E, E, E, E], [ir.Operand([(B, 0), (I, 1), (D, 2)], 3),
                                      ir.Operand([(B, 0), (J, 1), (D, 2)], 3)],
                       [ir.Output(B), ir.Output(I), ir.Output(J)], ir.RowValue(scores))
    return ir.Pipeline(producer, ir.Weight.exp(ir.Scale.over(h), ir.Shift.NONE), [], ir.Operand([(B, 0), (J, 1)], 2),
                       [B, I], ir.Normalizer.KEPT_GROUPS)


def smoother_tables(groups: int, nx: int, ny: int, seed: int = 0):
    """Device relations q (groups x nx positions), k (groups x ny) with x
    uniform[0, 1) (SplitMix64 salts 21, 22) and v (groups x ny) normal(0, 1)
    (salt 23), keys b, t (and d = 0) int64; and the x, y, v tensors."""
    import pyarrow as pa

    from . import kernels as K

    def table(n, salt, with_d=True):
        b = torch.arange(groups, dtype=torch.int64, device="cuda").repeat_interleave(n)
        t = torch.arange(n, dtype=torch.int64, device="cuda").repeat(groups)
        cols = [b, t] + ([torch.zeros_like(t)] if with_d else [])
        names = ["b", "t"] + (["d"] if with_d else []) + ["x"]
        x = S.units(seed, salt, groups * n) if with_d else S.normal(seed, salt, groups * n)
        schema = pa.schema([(c, pa.int64()) for c in names[:-1]] + [("x", pa.float64())])
        return K.DeviceRelation(schema, cols + [x]), x

    q, xs = table(nx, 21)
    k, ys = table(ny, 22)
    v, vs = table(ny, 23, with_d=False)
    return q, k, v, xs, ys, vs


def smoother(groups: int, nx: int, ny: int) -> None:
    from . import kernels as K

    q, k, v, _, _, _ = smoother_tables(groups, nx, ny)
    got = K.pipeline(smoother_pipeline(), [q, k, v], options=K.Options(result_on_device=True))
    rows = sum(batch.rows for batch in got.batches)
    for batch in got.batches:
        batch.release()
    print(f"smoother: {groups} groups x {nx} x {ny}: {rows} rows, {got.tiles_visited} tile pairs")


def main() -> None:
    p = argparse.ArgumentParser()
    sub = p.add_subparsers(dest="case", required=True)
    pa = sub.add_parser("attention")
    pa.add_argument("--groups", type=int, default=8)
    pa.add_argument("--t", type=int, default=2048)
    pa.add_argument("--d", type=int, default=64)
    pa.add_argument("--backward", action="store_true")
    pa.add_argument("--precision", choices=["split", "fp64"], default="split")
    pp = sub.add_parser("product")
    pp.add_argument("--n", type=int, default=4096)
    pg = sub.add_parser("ragged")
    pg.add_argument("--groups", type=int, default=64)
    pg.add_argument("--d", type=int, default=128)
    pg.add_argument("--window", type=int, default=512)
    pg.add_argument("--repeat", type=int, default=3)
    sub.add_parser("sparse")
    ps = sub.add_parser("smoother")
    ps.add_argument("--groups", type=int, default=64)
    ps.add_argument("--x", type=int, default=1 << 20)
    ps.add_argument("--y", type=int, default=256)
    pr = sub.add_parser("rank")
    pr.add_argument("--n", type=int, default=1 << 26)
    pr.add_argument("--repeat", type=int, default=3)
    args = p.parse_args()
    if args.case == "attention":
        attention(args.groups, args.t, args.d, args.backward,
                  Precision.FP64 if args.precision == "fp64" else Precision.SPLIT)
    elif args.case == "rank":
        rank(args.n, args.repeat)
    elif args.case == "ragged":
        ragged(args.groups, args.d, args.window, args.repeat)
    elif args.case == "sparse":
        sparse()
    elif args.case == "smoother":
        smoother(args.groups, args.x, args.y)
    else:
        product(args.n)


if __name__ == "__main__":
    main()
