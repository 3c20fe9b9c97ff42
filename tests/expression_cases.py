"""The cases of the reference's expression property
(crates/einfold-kernels/tests/expression_vs_sql.rs), drawn as it draws them:
two tables a(k, x, y) and b(k, x, y) of up to eight rows of DOUBLE values,
among them NULL, NaN, ±inf, ±0, ±1, ±800, 1e-300 and 1e300, and a random
expression of up to five levels over every operator, from the pinned
SplitMix64 stream in the reference's draw order."""
import math

from einfold_b200 import ir
from oracle import oracle

SEED, CASES = 0xE4E5, 300
SPECIAL = [math.nan, math.inf, -math.inf, 0.0, -0.0, 1.0, -1.0, 800.0, -800.0, 1e-300, 1e300]


def value(rng):
    r = rng.below(10)
    if r == 0:
        return None
    if r in (1, 2):
        return SPECIAL[rng.below(len(SPECIAL))]
    return (rng.unit() - 0.5) * 20.0


def expression(rng, depth):
    leaf = depth == 0 or rng.below(4) == 0
    if leaf:
        n = rng.below(5)
        if n == 0:
            return ir.Expression.literal([0.0, 1.0, 2.0, -0.5, 0.25, 3.5][rng.below(6)])
        operand = [0, 1][n % 2]
        column = [1, 2][n // 3]
        return ir.Expression.column(operand, column)
    n = rng.below(9)
    if n <= 3:
        op = [ir.Binary.ADD, ir.Binary.SUBTRACT, ir.Binary.MULTIPLY, ir.Binary.DIVIDE][rng.below(4)]
        a = expression(rng, depth - 1)
        b = expression(rng, depth - 1)
        return a.binary(op, b)
    if n == 4:
        a = expression(rng, depth - 1)
        p = [1.0, 2.0, 3.0, 0.5, 1.5][rng.below(5)]
        return a.binary(ir.Binary.POWER, ir.Expression.literal(p))
    op = [ir.Unary.NEGATE, ir.Unary.ABS, ir.Unary.EXP, ir.Unary.LN][n - 5]
    return expression(rng, depth - 1).unary(op)


def table(rows, rng):
    return [[value(rng), value(rng)] for _ in range(rows)]


def cases():
    """(seed, rows of a, rows of b, expression) of each of the reference's
    cases, in order."""
    for i in range(CASES):
        seed = (SEED + i) & ((1 << 64) - 1)
        rng = oracle.Rng.seeded(seed, 0)
        rows_a = table(rng.below(9), rng)
        rows_b = table(rng.below(9), rng)
        yield seed, rows_a, rows_b, expression(rng, 5)
