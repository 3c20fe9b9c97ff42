"""Engine-independent descriptions of folds and fold pipelines.

A Python mirror of einfold's IR crate (``crates/einfold-ir``): the same types,
the same validity rules, the same names. The kernels read these descriptions
and marshal them into the plain C structs that ``include/einfold_b200.h``
declares (see ``einfold_b200/kernels.py``).

Reference: ``crates/einfold-ir/src/fold.rs:59-416`` (Fold, Operand, Key, Output,
Domain, Condition), ``crates/einfold-ir/src/pipeline.rs:63-320`` (Pipeline,
Weight, Scale, Shift, Normalizer) and ``crates/einfold-ir/src/expression.rs:57-204``
(Expression, Unary, Binary).
"""
from __future__ import annotations

import enum
import math
import struct
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple


class InvalidFold(ValueError):
    """A description that breaks a rule (``fold.rs:InvalidFold``)."""


class KeyEquality(enum.IntEnum):
    """How a dimension's keys are compared: ``=`` or ``IS NOT DISTINCT FROM``."""

    EQUAL = 0
    NOT_DISTINCT = 1


@dataclass(frozen=True)
class Dimension:
    equality: KeyEquality = KeyEquality.EQUAL


EQ = Dimension(KeyEquality.EQUAL)


@dataclass(frozen=True)
class Key:
    """Which column of an operand holds which dimension's keys."""

    dimension: int
    column: int


@dataclass(frozen=True)
class Operand:
    """One input of a fold: its key columns and its factor column, if any."""

    keys: Tuple[Key, ...]
    factor: Optional[int] = None

    def __init__(self, keys: Sequence[Key] | Sequence[Tuple[int, int]], factor: Optional[int] = None):
        ks = tuple(k if isinstance(k, Key) else Key(int(k[0]), int(k[1])) for k in keys)
        object.__setattr__(self, "keys", ks)
        object.__setattr__(self, "factor", factor)

    def column_of(self, dim: int) -> Optional[int]:
        for k in self.keys:
            if k.dimension == dim:
                return k.column
        return None


@dataclass(frozen=True)
class DomainKey:
    column: int
    equality: KeyEquality = KeyEquality.EQUAL


class Comparison(enum.IntEnum):
    LESS = 0
    LESS_OR_EQUAL = 1
    GREATER = 2
    GREATER_OR_EQUAL = 3

    def holds(self, left, right) -> bool:
        if self is Comparison.LESS:
            return left < right
        if self is Comparison.LESS_OR_EQUAL:
            return left <= right
        if self is Comparison.GREATER:
            return left > right
        return left >= right

    def mirrored(self) -> "Comparison":
        return {
            Comparison.LESS: Comparison.GREATER,
            Comparison.LESS_OR_EQUAL: Comparison.GREATER_OR_EQUAL,
            Comparison.GREATER: Comparison.LESS,
            Comparison.GREATER_OR_EQUAL: Comparison.LESS_OR_EQUAL,
        }[self]


_I64_MIN, _I64_MAX = -(1 << 63), (1 << 63) - 1


@dataclass(frozen=True)
class Condition:
    """``left <comparison> right + offset`` between two dimensions' keys."""

    left: int
    comparison: Comparison
    right: int
    offset: int = 0

    def holds(self, left: int, right: int) -> bool:
        # Worked in unbounded integers, as the reference works in i128.
        return self.comparison.holds(int(left), int(right) + int(self.offset))

    def mirrored(self) -> Optional["Condition"]:
        if -self.offset > _I64_MAX:
            return None
        return Condition(self.right, self.comparison.mirrored(), self.left, -self.offset)


@dataclass(frozen=True)
class Output:
    dimension: int
    domain_key: Optional[DomainKey] = None


@dataclass(frozen=True)
class Domain:
    """A left join of the fold's groups onto a domain relation."""

    carry: Tuple[int, ...] = ()
    missing: Optional[float] = None

    def __eq__(self, other):
        if not isinstance(other, Domain):
            return NotImplemented
        bits = lambda m: None if m is None else struct.pack("<d", m)
        return self.carry == other.carry and bits(self.missing) == bits(other.missing)

    def __hash__(self):
        return hash((self.carry, None if self.missing is None else struct.pack("<d", self.missing)))


# ---------------------------------------------------------------------------
# Expressions (crates/einfold-ir/src/expression.rs)
# ---------------------------------------------------------------------------


class Unary(enum.IntEnum):
    NEGATE = 0
    ABS = 1
    EXP = 2
    LN = 3

    def apply(self, x: float) -> float:
        if self is Unary.NEGATE:
            return -x
        if self is Unary.ABS:
            return abs(x)
        if self is Unary.EXP:
            try:
                return math.exp(x)
            except OverflowError:
                return math.inf
        # Rust's f64::ln: NaN below 0 and -inf at 0.
        if math.isnan(x) or x < 0:
            return math.nan
        if x == 0:
            return -math.inf
        if math.isinf(x):
            return math.inf
        return math.log(x)


class Binary(enum.IntEnum):
    ADD = 0
    SUBTRACT = 1
    MULTIPLY = 2
    DIVIDE = 3
    POWER = 4

    def apply(self, a: float, b: float) -> float:
        if self is Binary.ADD:
            return a + b
        if self is Binary.SUBTRACT:
            return a - b
        if self is Binary.MULTIPLY:
            return a * b
        if self is Binary.DIVIDE:
            if b == 0.0:
                if a == 0.0 or math.isnan(a):
                    return math.nan
                neg = (math.copysign(1.0, a) < 0) != (math.copysign(1.0, b) < 0)
                return -math.inf if neg else math.inf
            return a / b
        return _powf(a, b)


def _powf(a: float, b: float) -> float:
    """IEEE ``pow`` (C99 Annex F), which Rust's ``f64::powf`` calls."""
    try:
        return math.pow(a, b)
    except OverflowError:
        # Overflow: sign follows a negative base raised to an odd integer.
        if a < 0 and b == int(b) and int(b) % 2 == 1:
            return -math.inf
        return math.inf
    except ValueError:
        # Domain errors: a negative finite base to a non-integer power (NaN),
        # or zero to a negative power (infinity).
        if a == 0.0 and b < 0:
            if b == int(b) and int(b) % 2 == 1:
                return math.copysign(math.inf, a)
            return math.inf
        return math.nan


class Expression:
    """A ``DOUBLE`` expression of a joined row (``expression.rs:117-135``).

    Build with :meth:`column`, :meth:`literal`, :meth:`unary`, :meth:`binary`.
    """

    __slots__ = ("kind", "operand", "col", "value", "op", "args")

    def __init__(self, kind, operand=None, col=None, value=None, op=None, args=()):
        self.kind = kind  # "column" | "literal" | "unary" | "binary"
        self.operand = operand
        self.col = col
        self.value = value
        self.op = op
        self.args = tuple(args)

    @staticmethod
    def column(operand: int, column: int) -> "Expression":
        return Expression("column", operand=int(operand), col=int(column))

    @staticmethod
    def literal(x: float) -> "Expression":
        return Expression("literal", value=float(x))

    def unary(self, op: Unary) -> "Expression":
        return Expression("unary", op=Unary(op), args=(self,))

    def binary(self, op: Binary, other: "Expression") -> "Expression":
        return Expression("binary", op=Binary(op), args=(self, other))

    def _identity(self):
        if self.kind == "column":
            return ("c", self.operand, self.col)
        if self.kind == "literal":
            return ("l", struct.pack("<d", self.value))
        return (self.kind[0], int(self.op)) + tuple(a._identity() for a in self.args)

    def __eq__(self, other):
        return isinstance(other, Expression) and self._identity() == other._identity()

    def __hash__(self):
        return hash(self._identity())

    def evaluate(self, column: Callable[[int, int], Optional[float]]) -> Optional[float]:
        """The expression's value; ``None`` (NULL) if any column it reads is NULL."""
        if self.kind == "column":
            return column(self.operand, self.col)
        if self.kind == "literal":
            return self.value
        if self.kind == "unary":
            x = self.args[0].evaluate(column)
            return None if x is None else self.op.apply(x)
        a = self.args[0].evaluate(column)
        b = self.args[1].evaluate(column)
        if a is None or b is None:
            return None
        return self.op.apply(a, b)

    def columns(self) -> List[Tuple[int, int]]:
        """Every column read, as ``(operand, column)``, in reading order."""
        out: List[Tuple[int, int]] = []

        def visit(e: "Expression"):
            if e.kind == "column":
                out.append((e.operand, e.col))
            for a in e.args:
                visit(a)

        visit(self)
        return out

    def postfix(self) -> List[Tuple[int, int, int, float]]:
        """The expression as postfix nodes ``(kind, op_or_operand, column, literal)``.

        Kinds: 0 column, 1 literal, 2 unary, 3 binary. This is the form the C
        ABI's ``einfold_expr_node`` array carries.
        """
        nodes: List[Tuple[int, int, int, float]] = []

        def visit(e: "Expression"):
            for a in e.args:
                visit(a)
            if e.kind == "column":
                nodes.append((0, e.operand, e.col, 0.0))
            elif e.kind == "literal":
                nodes.append((1, 0, 0, e.value))
            elif e.kind == "unary":
                nodes.append((2, int(e.op), 0, 0.0))
            else:
                nodes.append((3, int(e.op), 0, 0.0))

        visit(self)
        return nodes

    def __repr__(self):
        if self.kind == "column":
            return f"#{self.operand}.{self.col}"
        if self.kind == "literal":
            return repr(self.value)
        if self.kind == "unary":
            name = {Unary.NEGATE: "-", Unary.ABS: "abs", Unary.EXP: "exp", Unary.LN: "ln"}[self.op]
            return f"{name}({self.args[0]!r})"
        sym = {Binary.ADD: "+", Binary.SUBTRACT: "-", Binary.MULTIPLY: "*", Binary.DIVIDE: "/"}
        if self.op is Binary.POWER:
            return f"power({self.args[0]!r}, {self.args[1]!r})"
        return f"({self.args[0]!r} {sym[self.op]} {self.args[1]!r})"


class RowValue:
    """What each joined row contributes: the product of factors, or an expression."""

    PRODUCT: "RowValue"

    def __init__(self, expression: Optional[Expression] = None):
        self.expression = expression

    @property
    def is_product(self) -> bool:
        return self.expression is None

    def __eq__(self, other):
        return isinstance(other, RowValue) and self.expression == other.expression

    def __hash__(self):
        return hash(self.expression)

    def __repr__(self):
        return "Product" if self.is_product else f"Expression({self.expression!r})"


RowValue.PRODUCT = RowValue(None)


# ---------------------------------------------------------------------------
# Fold (crates/einfold-ir/src/fold.rs)
# ---------------------------------------------------------------------------


class Fold:
    """``SELECT outputs, SUM(row) FROM operands JOIN ... GROUP BY outputs``.

    Only ``SUM`` aggregates exist in the reference (``Aggregate::sum``), so the
    aggregate is implicit here.
    """

    def __init__(
        self,
        dimensions: Sequence[Dimension],
        operands: Sequence[Operand],
        outputs: Sequence[Output],
        row: RowValue = RowValue.PRODUCT,
        domain: Optional[Domain] = None,
        conditions: Sequence[Condition] = (),
    ):
        dimensions = list(dimensions)
        operands = list(operands)
        outputs = list(outputs)
        n = len(dimensions)
        for i, op in enumerate(operands):
            seen = [False] * n
            for k in op.keys:
                if k.dimension >= n or k.dimension < 0:
                    raise InvalidFold(f"operand {i} names dimension {k.dimension}, of {n}")
                if seen[k.dimension]:
                    raise InvalidFold(f"operand {i} holds dimension {k.dimension} twice")
                seen[k.dimension] = True
        for d in range(n):
            if not any(op.column_of(d) is not None for op in operands):
                raise InvalidFold(f"no operand holds dimension {d}")
        if row.is_product:
            if all(op.factor is None for op in operands):
                raise InvalidFold("no operand has a factor")
        else:
            for o, _ in row.expression.columns():
                if o >= len(operands):
                    raise InvalidFold(f"the row expression reads operand {o}, of {len(operands)}")
        seen = [False] * n
        for o in outputs:
            d = o.dimension
            if d >= n or d < 0:
                raise InvalidFold(f"output dimension {d}, of {n}")
            if seen[d]:
                raise InvalidFold(f"dimension {d} is output twice")
            seen[d] = True
            if (o.domain_key is not None) != (domain is not None):
                raise InvalidFold(
                    f"output of dimension {d} has a domain key exactly when the fold has a domain"
                )
        self._dimensions = dimensions
        self._operands = operands
        self._outputs = outputs
        self._row = row
        self._domain = domain
        self._conditions: List[Condition] = []
        if conditions:
            self._set_conditions(list(conditions))

    @classmethod
    def try_new(cls, dimensions, operands, outputs, row=RowValue.PRODUCT, domain=None) -> "Fold":
        return cls(dimensions, operands, outputs, row, domain)

    def _set_conditions(self, conditions: List[Condition]):
        n = len(self._dimensions)
        for c in conditions:
            if c.left >= n or c.right >= n:
                raise InvalidFold(f"a condition compares dimensions {c.left} and {c.right}, of {n}")
            if c.left == c.right:
                raise InvalidFold(f"a condition compares dimension {c.left} with itself")
        self._conditions = conditions

    def with_conditions(self, conditions: Sequence[Condition]) -> "Fold":
        f = Fold(self._dimensions, self._operands, self._outputs, self._row, self._domain)
        f._set_conditions(list(conditions))
        return f

    def dimensions(self) -> List[Dimension]:
        return self._dimensions

    def dimension(self, d: int) -> Dimension:
        return self._dimensions[d]

    def dimension_ids(self):
        return range(len(self._dimensions))

    def operands(self) -> List[Operand]:
        return self._operands

    def outputs(self) -> List[Output]:
        return self._outputs

    def row(self) -> RowValue:
        return self._row

    def domain(self) -> Optional[Domain]:
        return self._domain

    def conditions(self) -> List[Condition]:
        return self._conditions

    def output_of(self, dim: int) -> Optional[int]:
        for i, o in enumerate(self._outputs):
            if o.dimension == dim:
                return i
        return None

    def is_aggregated(self, dim: int) -> bool:
        return self.output_of(dim) is None

    def is_einsum(self) -> bool:
        return self._row.is_product


# ---------------------------------------------------------------------------
# Pipeline (crates/einfold-ir/src/pipeline.rs)
# ---------------------------------------------------------------------------


class Scale:
    """How a producer value ``p`` becomes a score: ``p``, ``p * c`` or ``p / c``."""

    def __init__(self, kind: int = 0, c: float = 1.0):
        self.kind = kind  # 0 one, 1 times, 2 over
        self.c = float(c)

    @staticmethod
    def one() -> "Scale":
        return Scale(0, 1.0)

    @staticmethod
    def times(c: float) -> "Scale":
        return Scale(1, c)

    @staticmethod
    def over(c: float) -> "Scale":
        return Scale(2, c)

    def apply(self, p: float) -> float:
        if self.kind == 0:
            return p
        if self.kind == 1:
            return p * self.c
        return Binary.DIVIDE.apply(p, self.c)

    def _identity(self):
        return (self.kind, struct.pack("<d", self.c) if self.kind else b"")

    def __eq__(self, other):
        return isinstance(other, Scale) and self._identity() == other._identity()

    def __hash__(self):
        return hash(self._identity())


class Shift(enum.IntEnum):
    NONE = 0
    KEPT_MAXIMUM = 1


class Normalizer(enum.IntEnum):
    KEPT_GROUPS = 0
    JOINED_ROWS = 1
    NONE = 2


class Weight:
    """A softmax weight ``exp(scale(p) - shift)`` or an expression of the score."""

    def __init__(self, scale: Optional[Scale] = None, shift: Shift = Shift.KEPT_MAXIMUM,
                 of: Optional[Expression] = None):
        self.scale = scale
        self.shift = shift
        self.of = of

    @staticmethod
    def exp(scale: Optional[Scale] = None, shift: Shift = Shift.KEPT_MAXIMUM) -> "Weight":
        return Weight(scale=scale or Scale.one(), shift=shift)

    @staticmethod
    def of_expression(e: Expression) -> "Weight":
        return Weight(of=e)

    @property
    def is_exp(self) -> bool:
        return self.of is None


class Pipeline:
    """A producer fold whose values a softmax (or other weight) averages over."""

    def __init__(self, producer: Fold, weight: Weight, dimensions: Sequence[Dimension],
                 values: Operand, outputs: Sequence[int], normalizer: Normalizer):
        row = producer.row()
        if producer.domain() is not None:
            raise InvalidFold(
                "a pipeline's producer is a SUM of products or of a row expression, with no domain")
        if not weight.is_exp:
            if any(c != (0, 0) for c in weight.of.columns()):
                raise InvalidFold("a pipeline's weight reads only the producer's value")
        if values.factor is None:
            raise InvalidFold("a pipeline's values operand has no factor")
        own = len(producer.dimensions())
        n = own + len(dimensions)
        produced = lambda d: producer.output_of(d) is not None
        held = [False] * n
        for key in values.keys:
            d = key.dimension
            if d >= n or (d < own and not produced(d)):
                raise InvalidFold(f"the values operand holds dimension {d}, not an output")
            if held[d]:
                raise InvalidFold(f"the values operand holds dimension {d} twice")
            held[d] = True
        output = [False] * n
        for d in outputs:
            if d >= n or (d < own and not produced(d)):
                raise InvalidFold(f"output dimension {d} is not a producer output")
            if output[d]:
                raise InvalidFold(f"dimension {d} is output twice")
            output[d] = True
        for o in producer.outputs():
            d = o.dimension
            if not output[d] and not held[d]:
                raise InvalidFold(f"producer output {d} is summed but not joined")
        for d in range(own, n):
            if not held[d]:
                raise InvalidFold(f"the values operand doesn't hold dimension {d}")
        del row
        self._producer = producer
        self._weight = weight
        self._dimensions = list(dimensions)
        self._values = values
        self._outputs = list(outputs)
        self._normalizer = Normalizer(normalizer)

    def producer(self) -> Fold:
        return self._producer

    def weight(self) -> Weight:
        return self._weight

    def dimensions(self) -> List[Dimension]:
        return self._dimensions

    def values(self) -> Operand:
        return self._values

    def outputs(self) -> List[int]:
        return self._outputs

    def normalizer(self) -> Normalizer:
        return self._normalizer

    def is_summed(self, d: int) -> bool:
        return self._producer.output_of(d) is not None and d not in self._outputs
