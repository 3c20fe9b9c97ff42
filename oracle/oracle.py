"""ORACLE — test infrastructure, not product code.

A CPU restatement of einfold's kernel layer (``crates/einfold-kernels``): the
control logic of ``dense::fold``, ``discriminate::fold``, ``fused::pipeline``,
``chain::fold`` and ``schema`` in Python over pyarrow and numpy, with the inner
loops in ``einfold_oracle.c`` (built to ``oracle/libeinfold_oracle.so``).

Only ``tests/``, ``__graft_entry__.smoke()`` (to check its result) and ``bench.py``'s
CPU-baseline leg may import this module. The product path never does.

Parity pins: the SplitMix64 known answers (``rng.rs:66-78``), the tile-visit
counts (``pipeline_vs_sql.rs:734-765``), the ``Bounds`` decline cases
(``fused.rs:1116-1177``), signed-zero keys (``keys.rs:83-93``), long-prefix
byte order (``discriminate.rs:663-683``) and the summation bounds of
``gemm.rs:52-89`` and ``kernels_vs_sql.rs:21-23`` are checked in
``tests/test_oracle.py``. Dense and discrimination sums follow the reference's
order with unfused multiply and add, so they are the reference's bits; the
fused tile's block products are pinned by tolerance (the reference calls the
``matrixmultiply`` crate there, whose bits depend on the CPU).
"""
from __future__ import annotations

import ctypes
import math
import os
import struct
import sys
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from einfold_b200 import ir  # noqa: E402  (the IR types are plain data)

LIB_PATH = os.path.join(_HERE, "libeinfold_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compiles the C restatement with gcc (no build system needed)."""
    src = os.path.join(_HERE, "einfold_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        cmd = (f"gcc -O3 -march=x86-64-v3 -ffp-contract=off -fno-fast-math -fPIC -shared -pthread "
               f"-o {LIB_PATH} {src} -lm")
        if os.system(cmd) != 0:
            raise RuntimeError("building the oracle failed: " + cmd)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.ef_rng_next.restype = ctypes.c_uint64
        _lib.ef_rng_seeded.restype = ctypes.c_uint64
        _lib.ef_rng_seeded.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        _lib.ef_ranks_of_words.restype = ctypes.c_int64
        _lib.ef_ranks_of_bytes.restype = ctypes.c_int64
        _lib.ef_gustavson.restype = ctypes.c_int64
        _lib.ef_fused.restype = ctypes.c_int64
        _lib.ef_bounds_hold.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


# ---------------------------------------------------------------------------
# SplitMix64 (crates/einfold-testkit/src/rng.rs)
# ---------------------------------------------------------------------------

_M64 = (1 << 64) - 1


class Rng:
    """SplitMix64 as ``einfold_testkit::Rng``: ``seeded(seed, salt)``."""

    def __init__(self, seed: int = 0, salt: int = 0):
        self.state = ((seed * 0x2545F4914F6CDD1D) & _M64) ^ salt

    @classmethod
    def seeded(cls, seed: int, salt: int) -> "Rng":
        return cls(seed, salt)

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _M64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        return z ^ (z >> 31)

    def below(self, n: int) -> int:
        return self.next_u64() % max(n, 1)

    def chance(self, p: float) -> bool:
        return self.unit() < p

    def unit(self) -> float:
        return (self.next_u64() >> 11) / float(1 << 53)

    def pick(self, xs):
        return xs[self.below(len(xs))]

    def shuffle(self, xs: list):
        for i in range(len(xs) - 1, 0, -1):
            j = self.below(i + 1)
            xs[i], xs[j] = xs[j], xs[i]

    # Bulk draws through the C restatement (same stream).
    def u64s(self, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.uint64)
        st = ctypes.c_uint64(self.state)
        lib().ef_rng_fill(ctypes.byref(st), _p(out), ctypes.c_int64(n))
        self.state = st.value
        return out

    def units(self, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float64)
        st = ctypes.c_uint64(self.state)
        lib().ef_rng_units(ctypes.byref(st), _p(out), ctypes.c_int64(n))
        self.state = st.value
        return out


# ---------------------------------------------------------------------------
# Options (crates/einfold-kernels/src/options.rs)
# ---------------------------------------------------------------------------

BITWISE, SIGNED_ZEROS_EQUAL = 0, 1


@dataclass
class Options:
    float_keys: int = BITWISE
    threads: int = 1
    unique_domain: bool = False


class Declined(Exception):
    pass


class MemoryError_(Exception):
    pass


@dataclass
class Folded:
    algorithm: str
    batches: List[pa.RecordBatch]


@dataclass
class Piped:
    batches: List[pa.RecordBatch]
    tiles_visited: int
    tiles: int


# ---------------------------------------------------------------------------
# Schemas (crates/einfold-kernels/src/schema.rs)
# ---------------------------------------------------------------------------


def schema(fold: ir.Fold, operands: Sequence[pa.Schema], domain: Optional[pa.Schema] = None) -> pa.Schema:
    if not fold.is_einsum():
        raise ValueError("EinFold computes SUM of products only")
    return _fold_schema(fold, operands, domain)


def _fold_schema(fold, operands, domain):
    chain = len(fold.operands()) == 3 and fold.domain() is None
    if not (len(fold.operands()) == 2 or chain) or len(operands) != len(fold.operands()):
        raise ValueError("EinFold computes folds of two operands, or chains of three")
    if (fold.domain() is not None) != (domain is not None):
        raise ValueError("a domain relation must be given exactly when the fold has a domain")

    def field(s: pa.Schema, col: int) -> pa.Field:
        if col >= len(s):
            raise ValueError(f"column {col} of an input with {len(s)}")
        return s.field(col)

    if fold.row().is_product:
        values = []
        for o, op in enumerate(fold.operands()):
            if op.factor is None:
                raise ValueError("EinFold doesn't compute masks yet")
            values.append((o, op.factor))
    else:
        values = fold.row().expression.columns()
    for o, c in values:
        if field(operands[o], c).type != pa.float64():
            raise ValueError("EinFold's values must be Float64")
    types: List[Optional[pa.Field]] = [None] * len(fold.dimensions())
    for op, s in zip(fold.operands(), operands):
        for k in op.keys:
            f = field(s, k.column)
            if types[k.dimension] is None:
                types[k.dimension] = f
            elif types[k.dimension].type != f.type:
                raise ValueError(f"dimension {k.dimension}'s columns have different types")
    fields = []
    if fold.domain() is not None:
        for o in fold.outputs():
            key = field(domain, o.domain_key.column)
            if key.type != types[o.dimension].type:
                raise ValueError("the domain's key type differs from the operands'")
        for col in fold.domain().carry:
            f = field(domain, col)
            fields.append(pa.field(str(len(fields)), f.type, f.nullable))
    else:
        for o in fold.outputs():
            f = types[o.dimension]
            fields.append(pa.field(str(len(fields)), f.type, f.nullable))
    nullable = fold.domain() is None or fold.domain().missing is None
    fields.append(pa.field(str(len(fields)), pa.float64(), nullable))
    return pa.schema(fields)


def pipeline_schema(p: ir.Pipeline, inputs: Sequence[pa.Schema]) -> pa.Schema:
    producer = _fold_schema(p.producer(), inputs[:2], None)
    values = p.values()

    def column(c):
        if c >= len(inputs[2]):
            raise ValueError(f"column {c} of the values operand")
        return inputs[2].field(c)

    if column(values.factor).type != pa.float64():
        raise ValueError("EinFold factors must be Float64")

    def key(d):
        o = p.producer().output_of(d)
        if o is not None:
            return producer.field(o)
        return column(values.column_of(d))

    for k in values.keys:
        if key(k.dimension).type != column(k.column).type:
            raise ValueError(f"dimension {k.dimension}'s columns have different types")
    fields = []
    for d in p.outputs():
        f = key(d)
        fields.append(pa.field(str(len(fields)), f.type, f.nullable))
    fields.append(pa.field(str(len(fields)), pa.float64(), True))
    return pa.schema(fields)


# ---------------------------------------------------------------------------
# Dense fold (crates/einfold-kernels/src/dense.rs:176-578)
# ---------------------------------------------------------------------------

ABSENT, NULL, VALUED = 0, 1, 2
XB, YB, ZB, FEW_CELLS = 256, 2048, 4096, 4096
U32_MAX = (1 << 32) - 1
NO_GROUP = -1


def _is_integer(t: pa.DataType) -> bool:
    return pa.types.is_integer(t)


def dense_keys(column: pa.Array) -> Optional[Tuple[np.ndarray, int]]:
    """``dense::keys`` (dense.rs:97-111): non-negative i64 keys and extent."""
    if not _is_integer(column.type) or column.null_count > 0:
        return None
    if pa.types.is_uint64(column.type):
        raw = column.to_numpy(zero_copy_only=False).astype(np.uint64)
        if len(raw) and raw.max() >= np.uint64(1 << 63):
            return None  # the cast makes it NULL, and a NULL declines
        k = raw.astype(np.int64)
    else:
        k = column.to_numpy(zero_copy_only=False).astype(np.int64)
    lo = min(int(k.min()), 0) if len(k) else 0
    hi = int(k.max()) if len(k) else -1
    if lo < 0:
        return None
    if hi + 1 > (1 << 63) - 1:
        return None
    return k, hi + 1


def _size(dims, extent):
    n = 1
    for d in dims:
        n *= extent[d]
        if n >= 1 << 64:
            return None
    return n


def _worth(cells: int, rows: int) -> bool:
    return cells <= rows * 4 + FEW_CELLS and cells < U32_MAX


def _positions(keys: dict, dims, extent, rows) -> np.ndarray:
    p = np.zeros(rows, dtype=np.uint64)
    for d in dims:
        p = p * np.uint64(extent[d]) + keys[d].astype(np.uint64)
    return p.astype(np.int64)


def _rows(batches) -> int:
    return sum(b.num_rows for b in batches)


def _factors(op: ir.Operand, batch: pa.RecordBatch):
    if op.factor is None:
        return None
    col = batch.column(op.factor)
    if col.type != pa.float64():
        return None
    return col


def _valid(col: pa.Array) -> np.ndarray:
    if col.null_count == 0:
        return np.ones(len(col), dtype=bool)
    return np.asarray(col.is_valid().to_numpy(zero_copy_only=False), dtype=bool)


def _values(col: pa.Array) -> np.ndarray:
    return np.asarray(col.fill_null(0.0).to_numpy(zero_copy_only=False), dtype=np.float64)


def dense_fold(fold: ir.Fold, a: Sequence[pa.RecordBatch], b: Sequence[pa.RecordBatch],
               domain: Optional[Sequence[pa.RecordBatch]], out_schema: pa.Schema,
               options: Options = Options()) -> Optional[List[pa.RecordBatch]]:
    ops = fold.operands()
    if len(ops) != 2:
        return None
    op_a, op_b = ops
    ws, xs, ys, zs = [], [], [], []
    for o in fold.outputs():
        d = o.dimension
        ha, hb = op_a.column_of(d) is not None, op_b.column_of(d) is not None
        if ha and hb:
            ws.append(d)
        elif ha:
            xs.append(d)
        elif hb:
            ys.append(d)
        else:
            return None
    xs = ws + xs
    for d in fold.dimension_ids():
        if fold.is_aggregated(d):
            if op_a.column_of(d) is None or op_b.column_of(d) is None:
                return None
            zs.append(d)
    is_output = lambda d: d in xs or d in ys
    if not all(is_output(c.left) and is_output(c.right) for c in fold.conditions()):
        return None

    def integers(op, batches):
        if not batches:
            return True
        return all(_is_integer(batches[0].column(k.column).type) for k in op.keys)

    if not integers(op_a, a) or not integers(op_b, b):
        return None

    def cast_keys(op, batches):
        out = []
        for batch in batches:
            keys = {}
            exts = {}
            for k in op.keys:
                r = dense_keys(batch.column(k.column))
                if r is None:
                    return None
                keys[k.dimension], exts[k.dimension] = r
            out.append((keys, exts))
        return out

    a_keys, b_keys = cast_keys(op_a, a), cast_keys(op_b, b)
    if a_keys is None or b_keys is None:
        return None
    extent = [0] * len(fold.dimensions())
    for _, exts in a_keys + b_keys:
        for d, n in exts.items():
            extent[d] = max(extent[d], n)
    wzs = ws + zs
    nw, nx, nz, ny = (_size(ws, extent), _size(xs, extent), _size(zs, extent), _size(ys, extent))
    if None in (nw, nx, nz, ny):
        return None
    per_batch = nx // nw if nw else 0
    out_rows = _rows(domain) if domain is not None else nx * ny
    if not _worth(nx * nz, _rows(a)) or not _worth(nw * nz * ny, _rows(b)) or not _worth(nx * ny, out_rows):
        return None
    zero_default = fold.domain() is not None and fold.domain().missing is not None and \
        struct.pack("<d", fold.domain().missing) == struct.pack("<d", 0.0)

    a_matrix = np.zeros(nx * nz, dtype=np.float64)
    held = np.zeros(nx * nz, dtype=np.uint8)
    reached = np.zeros(nx, dtype=bool)
    valued = np.zeros(nx, dtype=bool)
    finite = True
    for batch, (keys, _) in zip(a, a_keys):
        fa = _factors(op_a, batch)
        if fa is None:
            return None
        n = batch.num_rows
        px = _positions(keys, xs, extent, n)
        pz = _positions(keys, zs, extent, n)
        p = px * nz + pz
        valid = _valid(fa)
        vals = _values(fa)
        # A repeated position, within the batch or with an earlier one, is a duplicate.
        if np.any(held[p] != ABSENT) or len(np.unique(p)) != len(p):
            return None
        held[p] = np.where(valid, VALUED, NULL)
        reached[px] = True
        a_matrix[p[valid]] = vals[valid]
        if valid.any():
            finite &= bool(np.all(np.isfinite(vals[valid])))
        np.logical_or.at(valued, px, valid)
    b_matrix = np.zeros(nw * nz * ny, dtype=np.float64)
    present = np.zeros(nw * nz * ny, dtype=bool)
    b_nulls = False
    for batch, (keys, _) in zip(b, b_keys):
        fb = _factors(op_b, batch)
        if fb is None:
            return None
        b_nulls |= fb.null_count > 0
        n = batch.num_rows
        pz = _positions(keys, wzs, extent, n)
        py = _positions(keys, ys, extent, n)
        p = pz * ny + py
        if np.any(present[p]) or len(np.unique(p)) != len(p):
            return None
        present[p] = True
        valid = _valid(fb)
        vals = _values(fb)
        b_matrix[p[valid]] = vals[valid]
    holes = b_nulls or not bool(present.all())
    if holes and (not zero_default or not finite):
        return None

    masked = bool(fold.conditions())
    order = xs + ys

    def stride_of(d):
        slot = order.index(d)
        s = 1
        for e in order[slot + 1:]:
            s *= extent[e]
        return s

    located = []
    if fold.domain() is not None and domain is not None:
        for batch in domain:
            cell = np.zeros(batch.num_rows, dtype=np.int64)
            bad = np.zeros(batch.num_rows, dtype=bool)
            for o in fold.outputs():
                d = o.dimension
                col = batch.column(o.domain_key.column)
                if not _is_integer(col.type):
                    col = pc.cast(col, pa.int64())
                if pa.types.is_uint64(col.type):
                    raw = col.fill_null(0).to_numpy(zero_copy_only=False)
                    big = raw >= np.uint64(1 << 63)
                    k = np.where(big, -1, raw.astype(np.int64))
                else:
                    k = col.fill_null(0).to_numpy(zero_copy_only=False).astype(np.int64)
                valid = _valid(col) if not pa.types.is_uint64(col.type) else (_valid(col) & (k >= 0))
                in_range = (k >= 0) & (k < extent[d]) & valid
                bad |= ~in_range
                cell = cell + np.where(in_range, k, 0) * stride_of(d)
            cell[bad] = NO_GROUP
            located.append(cell)
        if options.unique_domain:
            allc = np.concatenate(located) if located else np.zeros(0, np.int64)
            allc = allc[allc != NO_GROUP]
            if len(np.unique(allc)) != len(allc):
                return None

    out = np.zeros(nx * ny, dtype=np.float64)
    lib().ef_dense_accumulate(_p(a_matrix), _p(held), _p(b_matrix), ctypes.c_int64(nx), ctypes.c_int64(nz),
                              ctypes.c_int64(ny), ctypes.c_int64(per_batch), _p(out),
                              ctypes.c_int(max(options.threads, 1)))

    def key_at(d, x, y):
        role, pos = (xs, x) if d in xs else (ys, y)
        slot = role.index(d)
        s = 1
        for e in role[slot + 1:]:
            s *= extent[e]
        return (pos // s) % extent[d]

    def allowed_cells(cx: np.ndarray, cy: np.ndarray) -> np.ndarray:
        keep = np.ones(len(cx), dtype=bool)
        for c in fold.conditions():
            l = key_at(c.left, cx, cy).astype(object) if False else key_at(c.left, cx, cy)
            r = key_at(c.right, cx, cy)
            # Keys are below 2^32, so i64 holds right + offset only when the
            # offset is moderate; compare in Python integers otherwise.
            if abs(c.offset) < (1 << 60):
                keep &= _cmp(c.comparison, l.astype(np.int64), r.astype(np.int64) + c.offset)
            else:
                keep &= np.array([c.holds(int(li), int(ri)) for li, ri in zip(l, r)], dtype=bool)
        return keep

    if fold.domain() is not None and domain is not None:
        spec = fold.domain()
        batches = []
        for batch, cell in zip(domain, located):
            ok = cell != NO_GROUP
            c = np.where(ok, cell, 0)
            cx, cy = c // max(ny, 1), c % max(ny, 1)
            has = ok.copy()
            if not zero_default:
                has &= valued[cx] if nx else np.zeros(len(c), bool)
            if masked:
                has &= allowed_cells(cx, cy)
            vals = out[c] if len(out) else np.zeros(len(c))
            cols = [batch.column(i) for i in spec.carry]
            if spec.missing is not None:
                col = pa.array(np.where(has, vals, spec.missing), type=pa.float64())
            else:
                col = pa.array(vals, type=pa.float64(), mask=~has)
            cols.append(col)
            batches.append(pa.RecordBatch.from_arrays(cols, schema=out_schema))
        return batches
    if fold.domain() is not None or domain is not None:
        return None
    rows = np.nonzero(reached)[0]
    n = len(rows) * ny
    cx = np.repeat(rows, ny)
    cy = np.tile(np.arange(ny), len(rows))
    columns = []
    for o in fold.outputs():
        k = key_at(o.dimension, cx, cy).astype(np.int64)
        ty = out_schema.field(len(columns)).type
        columns.append(pc.cast(pa.array(k, type=pa.int64()), ty))
    vals = out[cx * ny + cy] if n else np.zeros(0)
    if bool(np.all(valued[rows])):
        columns.append(pa.array(vals, type=pa.float64()))
    else:
        columns.append(pa.array(vals, type=pa.float64(), mask=~valued[cx]))
    batch = pa.RecordBatch.from_arrays(columns, schema=out_schema)
    if not masked:
        return [batch]
    keep = allowed_cells(cx, cy)
    return [batch.filter(pa.array(keep))]


def _cmp(comparison, l, r):
    if comparison == ir.Comparison.LESS:
        return l < r
    if comparison == ir.Comparison.LESS_OR_EQUAL:
        return l <= r
    if comparison == ir.Comparison.GREATER:
        return l > r
    return l >= r


# ---------------------------------------------------------------------------
# Keys and ranks (keys.rs, discriminate.rs:73-292)
# ---------------------------------------------------------------------------


def host_keys(columns: Sequence[pa.Array], float_keys: int) -> List[pa.Array]:
    """``keys::host_keys``: -0.0 becomes 0.0 for plain float columns."""
    if float_keys == BITWISE:
        return list(columns)
    out = []
    for c in columns:
        t = c.type
        if pa.types.is_floating(t):
            width = {16: np.uint16, 32: np.uint32, 64: np.uint64}[t.bit_width]
            v = c.to_numpy(zero_copy_only=False)
            v = np.asarray(v, dtype={16: np.float16, 32: np.float32, 64: np.float64}[t.bit_width])
            bits = v.view(width)
            neg0 = bits == width(1 << (t.bit_width - 1))
            if neg0.any():
                v = v.copy()
                v[neg0] = 0.0
                c = pa.array(v, type=t, mask=~_valid(c) if c.null_count else None)
        out.append(c)
    return out


def _float_order(v: np.ndarray, bits: int) -> np.ndarray:
    ut = {16: np.uint16, 32: np.uint32, 64: np.uint64}[bits]
    u = v.view(ut).astype(np.uint64)
    sign = np.uint64(1 << (bits - 1))
    mask = np.uint64((1 << bits) - 1)
    return np.where(u & sign, (~u) & mask, u | sign)


def _encode_column(c: pa.Array) -> List[bytes]:
    """An order- and equality-preserving, prefix-free byte encoding of a column,
    in Arrow's default order (nulls first, ascending)."""
    if pa.types.is_dictionary(c.type):
        c = c.dictionary_decode()
    t = c.type
    valid = _valid(c)
    n = len(c)
    if pa.types.is_temporal(t) and not pa.types.is_interval(t):
        # Dates, times, timestamps and durations order as their integers.
        c = c.cast(pa.int32() if t.bit_width == 32 else pa.int64())
        t = c.type
    if pa.types.is_decimal(t) or pa.types.is_fixed_size_binary(t):
        # Arrow's row format: a decimal's two's complement big-endian with
        # the sign bit flipped; fixed-size binary as its bytes.
        w = t.byte_width
        raw = c.buffers()[1].to_pybytes() if n else b""
        vals = []
        for i in range(n):
            b = raw[(c.offset + i) * w:(c.offset + i + 1) * w]
            if pa.types.is_decimal(t):
                b = bytearray(b[::-1])
                b[0] ^= 0x80
                b = bytes(b)
            vals.append(b)
        return [(b"\x01" + vals[i]) if valid[i] else b"\x00" for i in range(n)]
    if pa.types.is_integer(t):
        v = c.fill_null(0).to_numpy(zero_copy_only=False)
        if pa.types.is_signed_integer(t):
            u = (v.astype(np.int64).view(np.uint64) ^ np.uint64(1 << 63))
        else:
            u = v.astype(np.uint64)
        raw = u.astype(">u8").tobytes()
        vals = [raw[8 * i:8 * i + 8] for i in range(n)]
    elif pa.types.is_floating(t):
        bits = t.bit_width
        v = np.asarray(c.fill_null(0).to_numpy(zero_copy_only=False),
                       dtype={16: np.float16, 32: np.float32, 64: np.float64}[bits])
        raw = _float_order(v, bits).astype(">u8").tobytes()
        vals = [raw[8 * i:8 * i + 8] for i in range(n)]
    elif pa.types.is_boolean(t):
        v = c.fill_null(False).to_numpy(zero_copy_only=False)
        vals = [b"\x01" if x else b"\x00" for x in v]
    elif pa.types.is_string(t) or pa.types.is_large_string(t) or pa.types.is_binary(t) or \
            pa.types.is_large_binary(t):
        py = c.to_pylist()
        vals = []
        for x in py:
            if x is None:
                vals.append(b"")
                continue
            bs = x.encode("utf-8") if isinstance(x, str) else bytes(x)
            vals.append(bs.replace(b"\x00", b"\x00\xff") + b"\x00\x00")
    else:
        raise TypeError(f"no key encoding for {t}")
    return [(b"\x01" + vals[i]) if valid[i] else b"\x00" for i in range(n)]


@dataclass
class Ranks:
    rank: np.ndarray  # u32 per row
    first: np.ndarray  # u32 per rank


def ranks_of_words(words: np.ndarray, threads: int = 1) -> Ranks:
    n = len(words)
    rank = np.zeros(n, dtype=np.uint32)
    first = np.zeros(n, dtype=np.uint32)
    if n == 0:
        return Ranks(rank, first[:0])
    w = np.ascontiguousarray(words, dtype=np.uint64)
    k = lib().ef_ranks_of_words(_p(w), ctypes.c_int64(n), ctypes.c_int(threads), _p(rank), _p(first))
    return Ranks(rank, first[:k].copy())


def ranks_of_bytes(keys: List[bytes]) -> Ranks:
    n = len(keys)
    rank = np.zeros(n, dtype=np.uint32)
    first = np.zeros(n, dtype=np.uint32)
    if n == 0:
        return Ranks(rank, first[:0])
    off = np.zeros(n + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(k) for k in keys])
    data = np.frombuffer(b"".join(keys) or b"\x00", dtype=np.uint8).copy()
    k = lib().ef_ranks_of_bytes(_p(data), _p(off), ctypes.c_int64(n), _p(rank), _p(first))
    return Ranks(rank, first[:k].copy())


def signed_words(c: pa.Array) -> Optional[np.ndarray]:
    """``rank_columns``' integer fast path (discriminate.rs:244-272)."""
    t = c.type
    if c.null_count:
        return None
    if pa.types.is_int64(t) or pa.types.is_int32(t):
        v = c.to_numpy(zero_copy_only=False).astype(np.int64)
        return v.view(np.uint64) ^ np.uint64(1 << 63)
    if pa.types.is_uint64(t) or pa.types.is_uint32(t):
        return c.to_numpy(zero_copy_only=False).astype(np.uint64)
    return None


def rank_columns(columns: Sequence[pa.Array], n: int, threads: int = 1) -> Ranks:
    """``rank_columns`` (discriminate.rs:240-277)."""
    if len(columns) == 1:
        w = signed_words(columns[0])
        if w is not None:
            return ranks_of_words(w, threads)
    if n == 0:
        return Ranks(np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    if not columns:
        return ranks_of_words(np.zeros(n, dtype=np.uint64), threads)
    encoded = [_encode_column(c) for c in columns]
    keys = [b"".join(parts) for parts in zip(*encoded)]
    return ranks_of_bytes(keys)


def _concat(parts: Sequence[Sequence[pa.Array]]) -> List[pa.Array]:
    width = len(parts[0]) if parts else 0
    out = []
    for c in range(width):
        arrs = [p[c] for p in parts]
        if any(pa.types.is_dictionary(a.type) for a in arrs):
            arrs = [a.dictionary_decode() if pa.types.is_dictionary(a.type) else a for a in arrs]
        out.append(pa.concat_arrays(arrs))
    return out


def _joinable(columns: Sequence[pa.Array], strict: Sequence[bool], n: int) -> np.ndarray:
    ok = np.ones(n, dtype=bool)
    for c, s in zip(columns, strict):
        if s:
            cc = c.dictionary_decode() if pa.types.is_dictionary(c.type) else c
            ok &= _valid(cc)
    return ok


def _counting(rows: np.ndarray, key: np.ndarray) -> np.ndarray:
    """A stable counting sort of ``rows`` by ``key[rows]``."""
    return rows[np.argsort(key[rows], kind="stable")]


def _break_ties(rows: np.ndarray, k1: np.ndarray, k2: np.ndarray, factors: pa.Array) -> np.ndarray:
    """``break_ties``: runs of equal (k1, k2) ordered by factor bits, NULL first."""
    if len(rows) < 2:
        return rows
    valid = _valid(factors)
    bits = np.asarray(factors.fill_null(0.0).to_numpy(zero_copy_only=False), dtype=np.float64).view(np.uint64)
    # A NULL sorts before every value: key (valid, bits).
    a, b = k1[rows], k2[rows]
    same_next = (a[1:] == a[:-1]) & (b[1:] == b[:-1])
    if not same_next.any():
        return rows
    run = np.concatenate([[0], np.cumsum(~same_next)])
    order = np.lexsort((bits[rows], valid[rows], run))
    return rows[order]


def discriminate_fold(fold: ir.Fold, a: pa.RecordBatch, b: pa.RecordBatch,
                      domain: Optional[Sequence[pa.RecordBatch]], out_schema: pa.Schema,
                      options: Options = Options()) -> List[pa.RecordBatch]:
    """``discriminate::fold`` (discriminate.rs:369-650)."""
    threads = max(options.threads, 1)
    na, nb = a.num_rows, b.num_rows
    nd = _rows(domain) if domain is not None else 0
    if max(na + nb, max(na, nb) + nd) >= 1 << 32:
        raise ValueError("EinFold's discrimination algorithm ranks at most 2^32 - 1 rows together")
    ops = fold.operands()
    shared = [d for d in fold.dimension_ids() if ops[0].column_of(d) is not None and ops[1].column_of(d) is not None]
    a_out = [i for i in range(len(fold.outputs())) if ops[0].column_of(fold.outputs()[i].dimension) is not None]
    b_out = [i for i in range(len(fold.outputs())) if i not in a_out]
    col = lambda op, batch, d: batch.column(ops[op].column_of(d))

    def outputs(op, batch, outs):
        return host_keys([col(op, batch, fold.outputs()[i].dimension) for i in outs], options.float_keys)

    def factors(op, batch):
        if ops[op].factor is None or batch.column(ops[op].factor).type != pa.float64():
            raise ValueError("factors must be Float64")
        return batch.column(ops[op].factor)

    a_f, b_f = factors(0, a), factors(1, b)
    strict = [fold.dimension(d).equality == ir.KeyEquality.EQUAL for d in shared]
    a_sh = host_keys([col(0, a, d) for d in shared], options.float_keys)
    b_sh = host_keys([col(1, b, d) for d in shared], options.float_keys)
    a_joins, b_joins = _joinable(a_sh, strict, na), _joinable(b_sh, strict, nb)
    z = rank_columns(_concat([a_sh, b_sh]) if shared else [], na + nb, threads)
    a_outputs, b_outputs = outputs(0, a, a_out), outputs(1, b, b_out)

    def domain_columns(outs):
        per = [host_keys([batch.column(fold.outputs()[i].domain_key.column) for i in outs], options.float_keys)
               for batch in domain]
        return _concat(per) if per and outs else []

    def with_domain(own, outs, n):
        if nd == 0:
            return rank_columns(own, n, threads)
        return rank_columns(_concat([own, domain_columns(outs)]) if outs else [], n + nd, threads)

    x = with_domain(a_outputs, a_out, na)
    y = with_domain(b_outputs, b_out, nb)
    nx, nz, ny = max(len(x.first), 1), max(len(z.first), 1), max(len(y.first), 1)
    zr = z.rank.astype(np.int64)
    a_z = zr[:na]
    b_z = zr[na:na + nb]
    xr, yr = x.rank.astype(np.int64), y.rank.astype(np.int64)
    a_rows = np.nonzero(a_joins)[0].astype(np.int64)
    a_rows = _counting(a_rows, a_z)
    a_rows = _counting(a_rows, xr[:na])
    a_rows = _break_ties(a_rows, xr[:na], a_z, a_f)
    b_rows = np.nonzero(b_joins)[0].astype(np.int64)
    b_rows = _counting(b_rows, yr[:nb])
    b_rows = _counting(b_rows, b_z)
    b_rows = _break_ties(b_rows, b_z, yr[:nb], b_f)
    a_start = np.zeros(nx + 1, dtype=np.int64)
    np.add.at(a_start, xr[a_rows] + 1, 1)
    a_start = np.cumsum(a_start)
    b_start = np.zeros(nz + 1, dtype=np.int64)
    np.add.at(b_start, b_z[b_rows] + 1, 1)
    b_start = np.cumsum(b_start)
    b_y = yr[b_rows].astype(np.uint32)
    b_valid = _valid(b_f)[b_rows].astype(np.uint8)
    b_vals = np.asarray(b_f.fill_null(0.0).to_numpy(zero_copy_only=False), np.float64)[b_rows]
    a_valid = _valid(a_f).astype(np.uint8)
    a_vals = np.asarray(a_f.fill_null(0.0).to_numpy(zero_copy_only=False), np.float64)
    pairs = int(np.sum(b_start[a_z[a_rows] + 1] - b_start[a_z[a_rows]])) if len(a_rows) else 0
    cap = max(min(pairs, nx * ny), 1)
    gx = np.zeros(cap, np.uint32)
    gy = np.zeros(cap, np.uint32)
    gs = np.zeros(cap, np.float64)
    gv = np.zeros(cap, np.uint8)
    a_rows32 = a_rows.astype(np.uint32)
    a_z32 = a_z.astype(np.uint32) if na else np.zeros(1, np.uint32)
    args = [_p(a_rows32 if len(a_rows32) else np.zeros(1, np.uint32)), _p(a_start), _p(a_z32),
            _p(a_vals if na else np.zeros(1)), _p(a_valid if na else np.zeros(1, np.uint8)), _p(b_start),
            _p(b_y if len(b_y) else np.zeros(1, np.uint32)), _p(b_vals if len(b_vals) else np.zeros(1)),
            _p(b_valid if len(b_valid) else np.zeros(1, np.uint8))]
    k = lib().ef_gustavson(*args, ctypes.c_int64(nx), ctypes.c_int64(ny), ctypes.c_int(threads),
                           ctypes.c_int64(cap), _p(gx), _p(gy), _p(gs), _p(gv))
    assert k >= 0, "group capacity"
    gx, gy, gs, gv = gx[:k], gy[:k], gs[:k], gv[:k].astype(bool)
    spec = fold.domain()
    if spec is None:
        a_take = x.first[gx] if k else np.zeros(0, np.uint32)
        b_take = y.first[gy] if k else np.zeros(0, np.uint32)
        columns = []
        for i in range(len(fold.outputs())):
            if i in a_out:
                c = a_outputs[a_out.index(i)].take(pa.array(a_take, type=pa.uint32()))
            else:
                c = b_outputs[b_out.index(i)].take(pa.array(b_take, type=pa.uint32()))
            columns.append(c)
        columns.append(pa.array(gs, type=pa.float64(), mask=~gv))
        return [pa.RecordBatch.from_arrays(columns, schema=out_schema)]
    if domain is None:
        raise ValueError("a fold with a domain was given no domain relation")
    group_start = np.zeros(nx + 1, dtype=np.int64)
    np.add.at(group_start, gx.astype(np.int64) + 1, 1)
    group_start = np.cumsum(group_start)
    strict_o = [fold.outputs()[i].domain_key.equality == ir.KeyEquality.EQUAL for i in range(len(fold.outputs()))]
    offset = 0
    out = []
    for batch in domain:
        n = batch.num_rows
        keys = [batch.column(fold.outputs()[i].domain_key.column) for i in range(len(fold.outputs()))]
        matches = _joinable(keys, strict_o, n)
        vals = np.zeros(n, np.float64)
        has = np.zeros(n, bool)
        for r in range(n):
            xi = int(xr[na + offset + r]) if len(a_out) else 0
            yi = int(yr[nb + offset + r]) if len(b_out) else 0
            if matches[r] and xi < nx:
                lo, hi = group_start[xi], group_start[xi + 1]
                j = lo + int(np.searchsorted(gy[lo:hi], yi))
                if j < hi and gy[j] == yi and gv[j]:
                    vals[r], has[r] = gs[j], True
        offset += n
        cols = [batch.column(c) for c in spec.carry]
        if spec.missing is not None:
            cols.append(pa.array(np.where(has, vals, spec.missing), type=pa.float64()))
        else:
            cols.append(pa.array(vals, type=pa.float64(), mask=~has))
        out.append(pa.RecordBatch.from_arrays(cols, schema=out_schema))
    return out


def _whole(batches: Sequence[pa.RecordBatch], s: pa.Schema) -> pa.RecordBatch:
    if not batches:
        return pa.RecordBatch.from_arrays([pa.array([], type=f.type) for f in s], schema=s)
    return pa.Table.from_batches(list(batches), schema=s).combine_chunks().to_batches()[0] \
        if sum(b.num_rows for b in batches) else pa.RecordBatch.from_arrays(
            [pa.array([], type=f.type) for f in s], schema=s)


def fold(f: ir.Fold, a_schema: pa.Schema, a: Sequence[pa.RecordBatch], b_schema: pa.Schema,
         b: Sequence[pa.RecordBatch], domain: Optional[Sequence[pa.RecordBatch]], out_schema: pa.Schema,
         options: Options = Options()) -> Folded:
    """``algorithm::fold`` (algorithm.rs:97-133)."""
    if options.unique_domain:
        raise ValueError("only fold_dense checks that a domain's keys are unique")
    dense = dense_fold(f, a, b, domain, out_schema, options)
    if dense is not None:
        return Folded("dense", dense)
    if f.conditions():
        raise ValueError("the discrimination algorithm computes no masks")
    return Folded("discriminate", discriminate_fold(f, _whole(a, a_schema), _whole(b, b_schema), domain,
                                                    out_schema, options))


# ---------------------------------------------------------------------------
# Fused pipeline (fused.rs:151-489, 624-664)
# ---------------------------------------------------------------------------


class _Node(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("op", ctypes.c_int32), ("col", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("lit", ctypes.c_double)]


def _nodes(e: ir.Expression, slot_of) -> Tuple[ctypes.Array, int]:
    post = e.postfix()
    arr = (_Node * max(len(post), 1))()
    for i, (kind, op, col, lit) in enumerate(post):
        if kind == 0:
            arr[i] = _Node(0, 0, slot_of((op, col)), 0, 0.0)
        elif kind == 1:
            arr[i] = _Node(1, 0, 0, 0, lit)
        else:
            arr[i] = _Node(kind, op, 0, 0, 0.0)
    return arr, len(post)


def _place(op: ir.Operand, batches, rows_dims, cols_dims, column, extent, keys_per_batch):
    rows, cols = _size(rows_dims, extent), _size(cols_dims, extent)
    if rows is None or cols is None:
        return None
    cells = rows * cols
    total = _rows(batches)
    if total != cells or cells >= U32_MAX:
        return None
    matrix = np.zeros(cells, np.float64)
    held = np.zeros(cells, bool)
    for batch, keys in zip(batches, keys_per_batch):
        f = batch.column(column)
        if f.type != pa.float64() or f.null_count > 0:
            return None
        n = batch.num_rows
        r = _positions(keys, rows_dims, extent, n)
        c = _positions(keys, cols_dims, extent, n)
        cell = r * cols + c
        if np.any(held[cell]) or len(np.unique(cell)) != len(cell):
            return None
        held[cell] = True
        matrix[cell] = f.to_numpy(zero_copy_only=False)
    return matrix


def pipeline(p: ir.Pipeline, q: Sequence[pa.RecordBatch], k: Sequence[pa.RecordBatch],
             v: Sequence[pa.RecordBatch], out_schema: pa.Schema, options: Options = Options()) -> Optional[Piped]:
    """``fused::pipeline`` (fused.rs:151-489)."""
    producer = p.producer()
    if len(producer.operands()) != 2:
        return None
    op_q, op_k = producer.operands()
    values = p.values()
    own = len(producer.dimensions())
    n = own + len(p.dimensions())
    holds = lambda op, d: op.column_of(d) is not None
    output = lambda d: d in p.outputs()
    ws, xs, es, js = [], [], [], []
    for d in range(own):
        produced = producer.output_of(d) is not None
        sig = (holds(op_q, d), holds(op_k, d), produced, output(d), holds(values, d))
        if sig == (True, True, True, True, True):
            ws.append(d)
        elif sig == (True, False, True, True, False):
            xs.append(d)
        elif sig == (True, True, False, False, False):
            es.append(d)
        elif sig == (False, True, True, False, True):
            js.append(d)
        else:
            return None
    ys = list(range(own, n))
    if not all(output(d) for d in ys):
        return None
    mask = []
    for c in producer.conditions():
        if len(xs) == 1 and len(js) == 1 and (c.left, c.right) == (xs[0], js[0]):
            mask.append(c)
        elif len(xs) == 1 and len(js) == 1 and (c.left, c.right) == (js[0], xs[0]):
            m = c.mirrored()
            if m is None:
                return None
            mask.append(m)
        else:
            return None
    local_xs, local_js = list(xs), list(js)
    xs = ws + xs
    js = ws + js
    row = producer.row()
    if row.is_product:
        if op_q.factor is None or op_k.factor is None:
            return None
        read = [(0, op_q.factor), (1, op_k.factor)]
    else:
        read = sorted(set(row.expression.columns()))
        if not all(any(o == oo for oo, _ in read) for o in range(2)):
            return None
    if values.factor is None:
        return None
    placements = []
    for o, c in read:
        if o == 0:
            placements.append((op_q, q, xs, es, c))
        else:
            placements.append((op_k, k, es, js, c))
    placements.append((values, v, js, ys, values.factor))
    extent = [0] * n
    all_keys = []
    for op, batches, _, _, _ in placements:
        per = []
        for batch in batches:
            keys = {}
            for key in op.keys:
                r = dense_keys(batch.column(key.column))
                if r is None:
                    return None
                keys[key.dimension] = r[0]
                extent[key.dimension] = max(extent[key.dimension], r[1])
            per.append(keys)
        all_keys.append(per)
    nx, ne, nj, ny = _size(xs, extent), _size(es, extent), _size(js, extent), _size(ys, extent)
    lnx, lnj = _size(local_xs, extent), _size(local_js, extent)
    if None in (nx, ne, nj, ny, lnx, lnj):
        return None
    matrices = []
    for (op, batches, rd, cd, column), keys in zip(placements, all_keys):
        m = _place(op, batches, rd, cd, column, extent, keys)
        if m is None:
            return None
        matrices.append(m)
    vmat = matrices.pop()
    if nx * ny >= U32_MAX:
        return None
    vv = vmat.reshape(nj, ny) if nj and ny else vmat.reshape(max(nj, 0), max(ny, 0))
    finite = np.all(np.isfinite(vv), axis=1).astype(np.uint8) if ny else np.ones(nj, np.uint8)
    absv = np.where(np.isfinite(vv), np.abs(vv), np.nan)
    with np.errstate(all="ignore"):
        largest = np.nan_to_num(np.nanmax(np.where(np.isnan(absv), -np.inf, absv), axis=1, initial=0.0),
                                nan=0.0) if ny else np.zeros(nj)
        nz_abs = np.where(np.isnan(absv) | (absv == 0.0), np.inf, absv)
        smallest = np.min(nz_abs, axis=1, initial=np.inf) if ny else np.full(nj, np.inf)
    largest = np.ascontiguousarray(np.maximum(largest, 0.0))
    smallest = np.ascontiguousarray(smallest)
    x_tiles = -(-nx // 64) if nx else 0
    tile_pairs = 0
    for t in range(x_tiles):
        x0, x1 = t * 64, min((t + 1) * 64, nx)
        start = x0 // lnx * lnj if lnx else 0
        end = (x1 - 1) // lnx * lnj + lnj if lnx else 0
        tile_pairs += -(-end // 64) - start // 64
    shape = (ctypes.c_int64 * 6)(nx, ne, nj, ny, max(lnx, 1), lnj)
    mask_cmp = (ctypes.c_int * max(len(mask), 1))(*[int(c.comparison) for c in mask])
    mask_off = (ctypes.c_int64 * max(len(mask), 1))(*[int(c.offset) for c in mask])
    w = p.weight()
    if w.is_exp:
        weight_kind, scale_kind, scale_c = 0, w.scale.kind, w.scale.c
        shifted = int(w.shift == ir.Shift.KEPT_MAXIMUM)
        wnodes, wn = (_Node * 1)(), 0
    else:
        weight_kind, scale_kind, scale_c, shifted = 1, 0, 1.0, 0
        wnodes, wn = _nodes(w.of, lambda oc: 0)
    out = np.zeros(max(nx * ny, 1), np.float64)
    overflowed = ctypes.c_int(0)
    keep = [vmat, vv, finite, largest, smallest, out]
    if row.is_product:
        qm, km = matrices
        keep += [qm, km]
        snodes, sn = (_Node * 1)(), 0
        mats = (ctypes.c_void_p * 1)()
        side = (ctypes.c_int * 1)()
        visited = lib().ef_fused(shape, weight_kind, scale_kind, ctypes.c_double(scale_c), shifted,
                                 int(p.normalizer()), wnodes, wn, 0, _p(qm), _p(km), snodes, sn, 0, mats, side,
                                 len(mask), mask_cmp, mask_off, _p(vmat), _p(finite), _p(largest), _p(smallest),
                                 _p(out), max(options.threads, 1), ctypes.byref(overflowed))
    else:
        slot = {oc: i for i, oc in enumerate(read)}
        snodes, sn = _nodes(row.expression, lambda oc: slot[oc])
        mats = (ctypes.c_void_p * len(read))(*[m.ctypes.data for m in matrices])
        side = (ctypes.c_int * len(read))(*[o for o, _ in read])
        keep += matrices
        visited = lib().ef_fused(shape, weight_kind, scale_kind, ctypes.c_double(scale_c), shifted,
                                 int(p.normalizer()), wnodes, wn, 1, None, None, snodes, sn, len(read), mats, side,
                                 len(mask), mask_cmp, mask_off, _p(vmat), _p(finite), _p(largest), _p(smallest),
                                 _p(out), max(options.threads, 1), ctypes.byref(overflowed))
    if overflowed.value:
        return None
    lo = np.zeros(nx, np.int64)
    hi = np.zeros(nx, np.int64)
    for x in range(nx):
        l, h = ctypes.c_int64(), ctypes.c_int64()
        lib().ef_fused_allowed((ctypes.c_int64 * 2)(max(lnx, 1), lnj), len(mask), mask_cmp, mask_off,
                               ctypes.c_int64(x), ctypes.byref(l), ctypes.byref(h))
        lo[x], hi[x] = l.value, h.value
    rows = np.nonzero((lo < hi) & (nj > 0))[0]
    cx = np.repeat(rows, ny)
    cy = np.tile(np.arange(ny), len(rows))
    columns = []
    for d in p.outputs():
        role, pos = (xs, cx) if d in xs else (ys, cy)
        slot_i = role.index(d)
        s = 1
        for e in role[slot_i + 1:]:
            s *= extent[e]
        kk = (pos // s) % extent[d]
        columns.append(pc.cast(pa.array(kk.astype(np.int64), type=pa.int64()), out_schema.field(len(columns)).type))
    columns.append(pa.array(out[cx * ny + cy] if len(cx) else np.zeros(0), type=pa.float64()))
    return Piped([pa.RecordBatch.from_arrays(columns, schema=out_schema)], int(visited), int(tile_pairs))


def bounds_hold(heaviest, lightest, largest, smallest, terms, z, results, special) -> bool:
    """``Bounds::hold`` (fused.rs:1058-1086), restated in C."""
    r = np.ascontiguousarray(results, dtype=np.float64)
    s = np.ascontiguousarray(special, dtype=np.uint8)
    return bool(lib().ef_bounds_hold(ctypes.c_double(heaviest), ctypes.c_double(lightest), ctypes.c_double(largest),
                                     ctypes.c_double(smallest), ctypes.c_int64(terms), ctypes.c_int(z is not None),
                                     ctypes.c_double(z if z is not None else 0.0), _p(r), _p(s),
                                     ctypes.c_int64(len(r))))


# ---------------------------------------------------------------------------
# Chains (chain.rs:64-288)
# ---------------------------------------------------------------------------

LARGEST_BOUND = 1.0715086071862673e301


def fold_chain(f: ir.Fold, operands: Sequence[Tuple[pa.Schema, Sequence[pa.RecordBatch]]], out_schema: pa.Schema,
               options: Options = Options()) -> Optional[List[pa.RecordBatch]]:
    ops = f.operands()
    chained = len(ops) == 3 and f.row().is_product and f.domain() is None and not f.conditions() and \
        all(op.factor is not None for op in ops)
    if not chained:
        return None
    bound = 1.0
    for op, (s, batches) in zip(ops, operands):
        largest, rows = 0.0, 0
        for batch in batches:
            c = batch.column(op.factor)
            if c.type != pa.float64():
                return None
            rows += batch.num_rows
            v = c.drop_null().to_numpy(zero_copy_only=False)
            if len(v):
                if not np.all(np.isfinite(v)):
                    return None
                largest = max(largest, float(np.max(np.abs(v))))
        bound *= largest * rows
    if not bound <= LARGEST_BOUND:
        return None
    extent = [0] * len(f.dimensions())
    for op, (s, batches) in zip(ops, operands):
        for batch in batches:
            for key in op.keys:
                r = dense_keys(batch.column(key.column))
                if r is None:
                    return None
                extent[key.dimension] = max(extent[key.dimension], r[1])
    dims = lambda op: sorted(k.dimension for k in op.keys)
    union = lambda a, b: sorted(set(a) | set(b))

    def kept(pair, rest):
        return [d for d in pair if f.output_of(d) is not None or ops[rest].column_of(d) is not None]

    def cost(pair, rest):
        x, y = pair
        pr = union(dims(ops[x]), dims(ops[y]))
        kp = kept(pr, rest)
        prod = lambda ds: math.prod(extent[d] for d in ds)
        return prod(pr) + prod(union(kp, dims(ops[rest])))

    shares = lambda x, y: any(d in dims(ops[y]) for d in dims(ops[x]))
    best = None
    for pair, rest in (((0, 1), 2), ((1, 2), 0), ((0, 2), 1)):
        if not shares(*pair):
            continue
        c = cost(pair, rest)
        if best is None or c < best[0]:
            best = (c, pair, rest)
    if best is None:
        return None
    _, (x, y), rest = best
    pr = union(dims(ops[x]), dims(ops[y]))
    kp = kept(pr, rest)

    def renumbered(op, local):
        return ir.Operand([ir.Key(local.index(kk.dimension), kk.column) for kk in op.keys], op.factor)

    of = lambda local: [f.dimension(d) for d in local]
    first = ir.Fold(of(pr), [renumbered(ops[x], pr), renumbered(ops[y], pr)],
                    [ir.Output(pr.index(d)) for d in kp])
    local = union(kp, dims(ops[rest]))
    t_op = ir.Operand([ir.Key(local.index(d), c) for c, d in enumerate(kp)], len(kp))
    second = ir.Fold(of(local), [t_op, renumbered(ops[rest], local)],
                     [ir.Output(local.index(o.dimension)) for o in f.outputs()])
    first_schema = schema(first, [operands[x][0], operands[y][0]])

    def either(fd, a, b, s):
        r = dense_fold(fd, a[1], b[1], None, s, options)
        if r is not None:
            return r
        oa, ob = fd.operands()
        swapped = ir.Fold(fd.dimensions(), [ob, oa], fd.outputs())
        return dense_fold(swapped, b[1], a[1], None, s, options)

    t = either(first, operands[x], operands[y], first_schema)
    if t is None:
        return None
    return either(second, (first_schema, t), operands[rest], out_schema)
