"""The reference's expression property (crates/einfold-kernels/tests/
expression_vs_sql.rs) on the device interpreter the tile kernels run
(``einfold_evaluate_pairs``): its 300 cases from its seed, drawn by the
pinned SplitMix64 generator in the reference's order, two tables of up to
eight rows of DOUBLE values among them NULL, NaN, ±inf, ±0, ±1, ±800,
1e-300 and 1e300, and a random expression of up to five levels over every
operator; and power of every pair of special values (the second test
there). The reference holds its ``Expression::evaluate`` to DataFusion's
SQL bit for bit; here the device's value of every pair of rows is held to
``ir.Expression.evaluate``, this package's restatement of it: NULL exactly
where a column read is NULL, and the same bits (any NaN for NaN) wherever
no exp, ln or power other than squaring lies upstream. Those three come
from the device's math library, within 1-2 ulp of the host's, so below them
a value must lie within twice a first-order bound of that difference as it
propagates (4 ulp for each exp and ln, 8 for each power)."""
import math
import struct

import numpy as np
import pytest

from einfold_b200 import ir, kernels as K
from tests import expression_cases as X

pytestmark = pytest.mark.gpu

U = 2.0 ** -53
TINY = 5e-324  # the least subnormal


def _bound(e, column):
    """(value, bound): ``evaluate``'s value and a first-order bound on how far
    the device's may lie from it (0: the same bits); inf where the bound
    doesn't hold (a pole, a large relative error, a special value below a
    transcendental)."""
    if e.kind == "column":
        v = column(e.operand, e.col)
        return v, 0.0
    if e.kind == "literal":
        return e.value, 0.0
    if e.kind == "unary":
        x, ex = _bound(e.args[0], column)
        if x is None:
            return None, 0.0
        v = e.op.apply(x)
        if e.op in (ir.Unary.NEGATE, ir.Unary.ABS):
            return v, ex
        if not math.isfinite(v) or not math.isfinite(x):
            # A special argument or result (C99's: NaN, ±inf, exp's overflow
            # and zero, ln of 0 and of negatives) from an exact argument.
            return v, (0.0 if ex == 0.0 else math.inf)
        if e.op is ir.Unary.EXP:
            return v, (abs(v) * (ex + 4 * U) + 4 * TINY if ex < 1e-3 else math.inf)
        # ln of a positive finite value
        if ex >= x / 2:
            return v, math.inf
        return v, ex / x + 4 * U * abs(v)
    a, ea = _bound(e.args[0], column)
    b, eb = _bound(e.args[1], column)
    if a is None or b is None:
        return None, 0.0
    v = e.op.apply(a, b)
    if ea == 0.0 and eb == 0.0 and (e.op is not ir.Binary.POWER or b == 2.0):
        return v, 0.0  # one IEEE operation on the same operands
    if math.isinf(ea) or math.isinf(eb) or not (math.isfinite(a) and math.isfinite(b) and math.isfinite(v)):
        return v, math.inf
    if e.op in (ir.Binary.ADD, ir.Binary.SUBTRACT):
        return v, ea + eb + U * abs(v)
    if e.op is ir.Binary.MULTIPLY:
        return v, abs(a) * eb + abs(b) * ea + ea * eb + U * abs(v)
    if e.op is ir.Binary.DIVIDE:
        if b == 0.0 or eb >= abs(b) / 2:
            return v, math.inf
        return v, (ea + abs(v) * eb) / abs(b) + U * abs(v)
    # power with a literal exponent (eb = 0)
    if b == 2.0:
        return v, 2 * abs(a) * ea + ea * ea + U * abs(v)
    if a == 0.0 or ea >= abs(a) / 2:
        return v, (8 * U * abs(v) if ea == 0.0 else math.inf)
    return v, abs(v) * (abs(b) * ea / abs(a) + 8 * U)


def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _device(e, a_rows, b_rows):
    import torch

    def pack(rows):
        n = max(len(rows), 1)
        vals = np.zeros((n, 3))
        valid = np.zeros((n, 3), dtype=np.uint8)
        valid[:, 0] = 1
        for i, (x, y) in enumerate(rows):
            for c, v in ((1, x), (2, y)):
                if v is not None:
                    vals[i, c] = v
                    valid[i, c] = 1
        return torch.from_numpy(vals).cuda(), torch.from_numpy(valid).cuda()

    a, av = pack(a_rows)
    b, bv = pack(b_rows)
    out, valid = K.evaluate_pairs(e, a[:len(a_rows)], av[:len(a_rows)], b[:len(b_rows)], bv[:len(b_rows)])
    return out.cpu().numpy(), valid.cpu().numpy()


def _check(e, rows_a, rows_b, where):
    got, got_valid = _device(e, rows_a, rows_b)
    assert got.shape == (len(rows_a), len(rows_b)), where
    exact = bounded = 0
    for i, ra in enumerate(rows_a):
        for j, rb in enumerate(rows_b):
            rows = [ra, rb]
            want, err = _bound(e, lambda o, c: rows[o][c - 1])
            assert bool(got_valid[i, j]) == (want is not None), f"{where} rows {(i, j)}: NULL differs"
            if want is None:
                continue
            g = float(got[i, j])
            if err == 0.0:
                same = (math.isnan(g) and math.isnan(want)) or _bits(g) == _bits(want)
                assert same, f"{where} rows {(i, j)}: device {g!r}, evaluate {want!r}\n{e!r}"
                exact += 1
            elif math.isfinite(err):
                assert math.isfinite(g) and abs(g - want) <= 2 * err, \
                    f"{where} rows {(i, j)}: device {g!r}, evaluate {want!r} (bound {err:.3g})\n{e!r}"
                bounded += 1
    return exact, bounded


def test_row_expressions_compute_what_evaluate_does():
    exact = bounded = pairs = 0
    for seed, rows_a, rows_b, e in X.cases():
        pairs += len(rows_a) * len(rows_b)
        if not rows_a or not rows_b:
            continue  # either table may be empty, and so the cross join
        x, b = _check(e, rows_a, rows_b, f"seed {seed}")
        exact += x
        bounded += b
    # Values are held to the bits where no transcendental lies upstream, the
    # rest to the bound.
    assert pairs > 1000 and exact > 0 and bounded > 0


def test_power_of_special_values_is_evaluates():
    specials = [None, math.nan, math.inf, -math.inf, 0.0, -0.0, -2.0, 0.5, 2.0]
    pairs = [[base, exponent] for base in specials for exponent in specials
             if not (base == 0.0 and exponent is not None and exponent < 0.0)]  # an error in SQL
    power = ir.Expression.column(0, 1).binary(ir.Binary.POWER, ir.Expression.column(0, 2))
    got, valid = _device(power, pairs, [[0.0, 0.0]])
    for k, (base, exponent) in enumerate(pairs):
        want = power.evaluate(lambda o, c: [base, exponent][c - 1])
        assert bool(valid[k, 0]) == (want is not None), (base, exponent)
        if want is None:
            continue
        g = float(got[k, 0])
        if math.isnan(want) or math.isinf(want) or want == 0.0 or exponent == 2.0 or abs(want) == 1.0:
            # Special and exact results: the same bits.
            assert (math.isnan(g) and math.isnan(want)) or _bits(g) == _bits(want), (base, exponent, g, want)
        else:
            assert abs(g - want) <= 8 * U * abs(want), (base, exponent, g, want)
