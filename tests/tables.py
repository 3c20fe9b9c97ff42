"""Synthetic tables and comparison helpers for the parity tests."""
from __future__ import annotations

import itertools
import json
import os
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import pyarrow as pa

from einfold_b200 import ir
from oracle import oracle

U = 2.0 ** -53  # unit roundoff of FP64


def complete(names: Sequence[str], extents: Sequence[int], values: np.ndarray, rng: oracle.Rng,
             key_type=pa.int64(), nulls: Optional[np.ndarray] = None, batches: int = 3,
             shuffle: bool = True) -> Tuple[pa.Schema, List[pa.RecordBatch]]:
    """A table with one row per key tuple, keys first-slowest, a value per row;
    rows shuffled and split into random batches."""
    n = int(np.prod(extents)) if extents else 1
    grids = np.indices(extents).reshape(len(extents), -1) if extents else np.zeros((0, 1), np.int64)
    order = np.arange(n)
    if shuffle and n > 1:
        perm = list(range(n))
        rng.shuffle(perm) if n <= 200_000 else None
        order = np.array(perm) if n <= 200_000 else np.argsort(rng.u64s(n), kind="stable")
    cols = [pa.array(grids[d][order], type=key_type) for d in range(len(extents))]
    v = np.asarray(values, dtype=np.float64).reshape(-1)[order]
    mask = None if nulls is None else np.asarray(nulls, bool).reshape(-1)[order]
    cols.append(pa.array(v, type=pa.float64(), mask=mask))
    schema = pa.schema([(nm, key_type) for nm in names] + [("v", pa.float64())])
    table = pa.Table.from_arrays(cols, schema=schema)
    out = []
    cuts = sorted(set([0, n] + [rng.below(n + 1) for _ in range(max(batches - 1, 0))]))
    for lo, hi in zip(cuts[:-1], cuts[1:]):
        out.extend(table.slice(lo, hi - lo).to_batches())
    if not out:
        out = [pa.RecordBatch.from_arrays([c.slice(0, 0) for c in cols], schema=schema)]
    return schema, out


def matmul_fold(domain: bool = False, missing: Optional[float] = None) -> ir.Fold:
    """SUM(a.v * b.v) over a(i, j) JOIN b(j, k) GROUP BY i, k."""
    e = ir.EQ
    if domain:
        return ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                       [ir.Output(0, ir.DomainKey(0)), ir.Output(2, ir.DomainKey(1))],
                       domain=ir.Domain((0, 1), missing))
    return ir.Fold([e, e, e], [ir.Operand([(0, 0), (1, 1)], 2), ir.Operand([(1, 0), (2, 1)], 2)],
                   [ir.Output(0), ir.Output(2)])


def rows_of(batches: Sequence[pa.RecordBatch]) -> pa.Table:
    if not batches:
        return None
    return pa.Table.from_batches(list(batches))


def split_bound(K: int, ma: np.ndarray, mb: np.ndarray, slices: int = 6) -> np.ndarray:
    """The split product's bound per cell: K terms, each within
    (8 + 16(S + 1))·2^-8S of the product of its row's and column's largest
    magnitudes (digit rounding plus the levels left out), plus the FP64
    combine's roundings."""
    return K * (8.0 + 16.0 * (slices + 1)) * 2.0 ** (-8 * slices) * np.outer(ma, mb)


def assert_same_rows(got: pa.Table, want: pa.Table, tol: Optional[np.ndarray] = None, exact: bool = False):
    """Same keys in the same order, same NULLs, values bit-exact or within `tol`."""
    assert got.num_rows == want.num_rows, (got.num_rows, want.num_rows)
    assert got.num_columns == want.num_columns
    for c in range(got.num_columns - 1):
        assert got.column(c).type == want.column(c).type, (got.column(c).type, want.column(c).type)
        gc, wc = got.column(c).combine_chunks(), want.column(c).combine_chunks()
        if pa.types.is_floating(gc.type):
            # By their bits, NaNs and signed zeros included.
            assert gc.null_count == wc.null_count and gc.is_null().equals(wc.is_null()), f"key column {c} NULLs differ"
            width = {16: np.uint16, 32: np.uint32, 64: np.uint64}[gc.type.bit_width]
            gb = np.asarray(gc.fill_null(0).to_numpy(zero_copy_only=False)).view(width)
            wb = np.asarray(wc.fill_null(0).to_numpy(zero_copy_only=False)).view(width)
            assert np.array_equal(gb, wb), f"key column {c} differs"
        else:
            assert gc.equals(wc), f"key column {c} differs"
    gv, wv = got.column(got.num_columns - 1), want.column(want.num_columns - 1)
    gnull = np.asarray(gv.is_null().to_numpy(zero_copy_only=False), bool)
    wnull = np.asarray(wv.is_null().to_numpy(zero_copy_only=False), bool)
    assert np.array_equal(gnull, wnull), "NULLs differ"
    g = np.asarray(gv.fill_null(0.0).to_numpy(zero_copy_only=False), np.float64)
    w = np.asarray(wv.fill_null(0.0).to_numpy(zero_copy_only=False), np.float64)
    if exact:
        same = (g.view(np.uint64) == w.view(np.uint64)) | (np.isnan(g) & np.isnan(w))
        assert same.all(), f"{(~same).sum()} values differ in bits; first at {np.nonzero(~same)[0][:5]}"
        return
    assert np.array_equal(np.isnan(g), np.isnan(w)), "NaNs differ"
    fin = np.isfinite(w)
    assert np.array_equal(g[~fin & ~np.isnan(w)], w[~fin & ~np.isnan(w)]), "infinities differ"
    err = np.abs(g[fin] - w[fin])
    if tol is None:
        assert (err == 0).all()
    else:
        t = np.broadcast_to(tol, w.shape)[fin]
        bad = err > t
        assert not bad.any(), f"{bad.sum()} values outside tolerance; worst {np.max(err - t)}"


def reference_facts() -> dict:
    """The reference's known answers, extracted from its sources by
    tests/golden/make_golden.py into tests/golden/reference_facts.json."""
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_facts.json")) as f:
        return json.load(f)
